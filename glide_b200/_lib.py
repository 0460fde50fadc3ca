"""ctypes binding of the C ABI in include/glide_b200.h (libglide_b200.so).

The product path has no CPU fallback: if the sm_100a library is missing or
fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "_lib" / "libglide_b200.so"

GLIDE_OK = 0
GLIDE_ERR_ARG = 1
GLIDE_ERR_SHAPE = 2
GLIDE_ERR_CUDA = 3
GLIDE_ERR_NONFINITE = 4
GLIDE_ERR_STATE = 5
GLIDE_ERR_NOT_CONVERGED = 6
GLIDE_ERR_TIMEOUT = 7
GLIDE_F64 = 0
GLIDE_F32 = 1
GLIDE_MIXED = 2

FIELDS = [
    "u", "v", "H", "H_prev", "phi", "mask", "bed", "B", "beta", "smb", "gamma",
    "f_u", "f_v", "f_H", "r_u", "r_v", "r_H",
    "lambda_u", "lambda_v", "lambda_H",
    "adj_f_u", "adj_f_v", "adj_f_H", "adj_r_u", "adj_r_v", "adj_r_H",
    "grad_beta", "grad_bed", "grad_H_prev", "grad_smb",
    "vjp_u", "vjp_v", "vjp_H",
    "F_u", "F_v", "F_H",
    "var_u", "var_v", "var_H", "jvp_u", "jvp_v", "jvp_H",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}

USE_MASK = 1
OPERATOR_ONLY = 2
FREEZE_CALVING = 4
FREEZE_PHI = 8

GRAD_BETA = 1
GRAD_BED = 2
GRAD_H_PREV = 4
GRAD_SMB = 8
GRAD_ALL = 15

MAX_HISTORY = 256

# glide_set_tuning keys (GLIDE_TUNE_*) and glide_group_set_tuning keys (GLIDE_GROUP_TUNE_*)
TUNE_SWEEP_BLOCKS_PER_SM = 1
TUNE_MIXED_INNER_VCYCLES = 2
TUNE_FORWARD_METHOD = 3
TUNE_NEWTON_SWITCH_EXP10 = 4
TUNE_TANGENT_VCYCLES = 5
TUNE_TMA_STAGING = 6
TUNE_REPORT_NOT_CONVERGED = 7
TUNE_TMA_GIVE_UP = 8
GROUP_TUNE_WAVES = 1
GROUP_TUNE_SPOIL_MAPS = 2

# glide_enthalpy_set_tuning keys (GLIDE_ENTH_TUNE_*) and enthalpy term bits (GLIDE_ENTH_*)
ENTH_TUNE_POINT_BLOCKS = 1
ENTH_TUNE_COLUMN_BLOCKS = 2
ENTH_TUNE_COLUMN_L1 = 3
ENTH_TUNE_COLUMN_KERNEL = 4
ENTH_HORIZ_ADV = 1
ENTH_SIGMA_DOT = 2
ENTH_DRAINAGE = 4
ENTH_MAX_HISTORY = 256

# glide_transfer op codes
TRANSFER_OPS = {
    "restrict_vfacet": 0, "restrict_hfacet": 1, "restrict_cell_avg": 2, "restrict_cell_max": 3,
    "restrict_cell_min": 4, "restrict_cell_var": 5,
    "prolongate_vfacet_injection": 6, "prolongate_vfacet_bilinear": 7,
    "prolongate_hfacet_injection": 8, "prolongate_hfacet_bilinear": 9,
    "prolongate_cell_injection": 10, "prolongate_cell_bilinear": 11,
    "prolongate_hfacet_as_vfacet_injection": 12, "prolongate_hfacet_as_vfacet_bilinear": 13,
}


class GlideError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"glide_b200 error {code}: {msg}")
        self.code = code


class NotConverged(GlideError):
    """A solve stopped at its cycle cap short of its tolerances (raised only
    when the handle reports it; every output is written).  `stats` holds the
    solve's statistics."""

    def __init__(self, msg, stats):
        super().__init__(GLIDE_ERR_NOT_CONVERGED, msg)
        self.stats = stats


class Phys(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "n", "eps_reg", "flotation_reg_driving", "m", "u_reg", "water_drag",
        "flotation_reg_sliding", "calving_rate", "flotation_reg_calving", "thklim")]


class FasConfig(ctypes.Structure):
    _fields_ = [("freeze_coarse_calving", ctypes.c_int), ("freeze_coarse_phi", ctypes.c_int),
                ("coarsest_steps", ctypes.c_int), ("pre_steps", ctypes.c_int),
                ("post_steps", ctypes.c_int), ("finest_steps", ctypes.c_int),
                ("maximum_vcycles", ctypes.c_int), ("relative_tolerance", ctypes.c_double),
                ("absolute_tolerance", ctypes.c_double)]


class VankaConfig(ctypes.Structure):
    _fields_ = [("omega", ctypes.c_double), ("newton_steps", ctypes.c_int),
                ("relaxation", ctypes.c_double), ("ssa_damping", ctypes.c_double),
                ("mc_damping", ctypes.c_double), ("relax_phi", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("vcycles", ctypes.c_int), ("initial_norm", ctypes.c_double),
                ("final_norm", ctypes.c_double), ("norms", ctypes.c_double * 3),
                ("history", ctypes.c_double * MAX_HISTORY)]

    def to_dict(self):
        n = self.vcycles
        return dict(vcycles=n, initial_norm=self.initial_norm, final_norm=self.final_norm,
                    norms=list(self.norms), history=list(self.history[: min(n + 1, MAX_HISTORY)]))


_H = ctypes.c_void_p
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

SIGNATURES = {
    "glide_last_error": ([], ctypes.c_char_p),
    "glide_version": ([], _I),
    "glide_create": ([_I, _I, _D, _I, _I, ctypes.POINTER(_H)], _I),
    "glide_destroy": ([_H], _I),
    "glide_level_shape": ([_H, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_D)], _I),
    "glide_field_ptr": ([_H, _I, _I, ctypes.POINTER(_P), ctypes.POINTER(_I), ctypes.POINTER(_I),
                         ctypes.POINTER(_I)], _I),
    "glide_set_field": ([_H, _I, _I, _P, _I, _I, _I, _P], _I),
    "glide_get_field": ([_H, _I, _I, _P, _I, _I, _P], _I),
    "glide_fill_field": ([_H, _I, _I, _D, _I, _P], _I),
    "glide_restrict_field": ([_H, _I, _I, _P], _I),
    "glide_set_phys": ([_H, _I, ctypes.POINTER(Phys)], _I),
    "glide_get_phys": ([_H, _I, ctypes.POINTER(Phys)], _I),
    "glide_set_fas_config": ([_H, _I, ctypes.POINTER(FasConfig)], _I),
    "glide_get_fas_config": ([_H, _I, ctypes.POINTER(FasConfig)], _I),
    "glide_set_vanka_config": ([_H, _I, _I, ctypes.POINTER(VankaConfig)], _I),
    "glide_get_vanka_config": ([_H, _I, _I, ctypes.POINTER(VankaConfig)], _I),
    "glide_set_reference_quirks": ([_H, _I], _I),
    "glide_set_use_graphs": ([_H, _I], _I),
    "glide_launch_count": ([_H, ctypes.POINTER(ctypes.c_longlong)], _I),
    "glide_alg_bytes": ([_H, ctypes.POINTER(ctypes.c_double)], _I),
    "glide_block_smoother_part": ([_H, _I, _D, _I, _I, _P], _I),
    "glide_set_tuning": ([_H, _I, _I], _I),
    "glide_set_rhs": ([_H, _I, _D, _P], _I),
    "glide_compute_phi": ([_H, _I, _D, _P], _I),
    "glide_residual": ([_H, _I, _D, _I, ctypes.POINTER(_D), _P], _I),
    "glide_vanka_sweep": ([_H, _I, _D, _I, _I, _P, _P], _I),
    "glide_vanka_dump": ([_H, _I, _D, _P, _P, _P], _I),
    "glide_forward": ([_H, _D, _I, ctypes.POINTER(Stats), _P], _I),
    "glide_adjoint_residual": ([_H, _I, _D, ctypes.POINTER(_D), _P], _I),
    "glide_vjp": ([_H, _I, _D, _P], _I),
    "glide_jvp": ([_H, _I, _D, _I, _I, _P], _I),
    "glide_adjoint_sweep": ([_H, _I, _D, _I, _P], _I),
    "glide_gradients": ([_H, _I, _D, _I, _P], _I),
    "glide_backward": ([_H, _D, _I, _I, ctypes.POINTER(Stats), _P], _I),
    "glide_residual_norms_noalloc": ([_I, _I, _D, _D, ctypes.POINTER(Phys), _P, _I, _P, _I, _P, _P, _P,
                                      _P, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P], _I),
    "glide_noalloc_last_error": ([], ctypes.c_char_p),
    "glide_vcycle": ([_H, _I, _I, _I, _D, _P], _I),
    "glide_transfer": ([_I, _I, _I, _I, _P, _I, _P, _I, _P], _I),
    "glide_group_create": ([ctypes.POINTER(_H), _I, ctypes.POINTER(_H)], _I),
    "glide_group_destroy": ([_H], _I),
    "glide_group_forward": ([_H, _D, _I, ctypes.POINTER(Stats), _P], _I),
    "glide_group_backward": ([_H, _D, _I, _I, ctypes.POINTER(Stats), _P], _I),
    "glide_group_counters": ([_H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_I)], _I),
    "glide_group_set_tuning": ([_H, _I, _I], _I),
}

class EnthalpyConfig(ctypes.Structure):
    _fields_ = [("omega", ctypes.c_double), ("n_newton", ctypes.c_int), ("relaxation", ctypes.c_double),
                ("relative_tolerance", ctypes.c_double), ("absolute_tolerance", ctypes.c_double),
                ("lf_c", ctypes.c_double), ("drain_rate", ctypes.c_double), ("h_thin", ctypes.c_double),
                ("term_flags", ctypes.c_int)]


class EnthalpyInputs(ctypes.Structure):
    _fields_ = [("H", ctypes.c_void_p), ("ld_H", ctypes.c_int), ("u", ctypes.c_void_p), ("ld_u", ctypes.c_int),
                ("u_layer", ctypes.c_longlong), ("v", ctypes.c_void_p), ("ld_v", ctypes.c_int),
                ("v_layer", ctypes.c_longlong), ("vel_div", ctypes.c_double)]


class EnthalpyStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("initial_norm", ctypes.c_double), ("final_norm", ctypes.c_double),
                ("history", ctypes.c_double * 256)]


SIGNATURES.update({
    "glide_enthalpy_last_error": ([], ctypes.c_char_p),
    "glide_enthalpy_create": ([_I, _I, _I, _D, ctypes.POINTER(_H)], _I),
    "glide_enthalpy_destroy": ([_H], _I),
    "glide_enthalpy_field_ptr": ([_H, _I, ctypes.POINTER(_P)], _I),
    "glide_enthalpy_set_config": ([_H, ctypes.POINTER(EnthalpyConfig)], _I),
    "glide_enthalpy_get_config": ([_H, ctypes.POINTER(EnthalpyConfig)], _I),
    "glide_enthalpy_set_inputs": ([_H, ctypes.POINTER(EnthalpyInputs)], _I),
    "glide_enthalpy_set_tuning": ([_H, _I, _I], _I),
    "glide_enthalpy_snapshot": ([_H, _P], _I),
    "glide_enthalpy_set_rhs": ([_H, _P], _I),
    "glide_enthalpy_residual": ([_H, _D, _I, ctypes.POINTER(_D), _P], _I),
    "glide_enthalpy_column_smooth": ([_H, _D, _P], _I),
    "glide_enthalpy_layer_smooth": ([_H, _D, _P], _I),
    "glide_enthalpy_column_sweep": ([_H, _D, _I, _I, ctypes.POINTER(EnthalpyStats), _P], _I),
    "glide_enthalpy_compute_omega": ([_H, _P, _I, _P, _I, _D, _D, _P], _I),
    "glide_enthalpy_frictional_heating": ([_H, _P, _I, _D, _D, _P], _I),
    "glide_enthalpy_arrhenius": ([_H, _D, _D, _P, _I, _P], _I),
    "glide_enthalpy_counters": ([_H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)], _I),
})



class VtiComponent(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int), ("kind", ctypes.c_int),
                ("stride_i", ctypes.c_longlong), ("stride_j", ctypes.c_longlong), ("stride_k", ctypes.c_longlong)]


class VtiArray(ctypes.Structure):
    _fields_ = [("n_components", ctypes.c_int), ("comp", VtiComponent * 3)]


VTI_MAX_ARRAYS = 16
VTI_PLAIN, VTI_XFACE, VTI_YFACE = 0, 1, 2

SIGNATURES.update({
    "glide_vti_pack": ([_I, _I, _I, _I, ctypes.POINTER(VtiArray), _I, _P, ctypes.c_size_t,
                        ctypes.POINTER(ctypes.c_size_t), _P], _I),
    "glide_io_last_error": ([], ctypes.c_char_p),
})

_LIB = None


def load(path: str | os.PathLike | None = None):
    """Load libglide_b200.so (once) and declare every exported signature."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise GlideError(GLIDE_ERR_STATE, f"{p} is missing; build it with `python -m glide_b200.build`")
    lib = ctypes.CDLL(str(p))
    for name, (argtypes, restype) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    if path is None:
        _LIB = lib
    return lib


def check(code: int):
    if code != GLIDE_OK:
        msg = load().glide_last_error()
        raise GlideError(code, msg.decode() if msg else "")


def call(name: str, *args):
    check(getattr(load(), name)(*args))
