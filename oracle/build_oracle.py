"""Build recipe for the CPU oracle (test infrastructure only).

Outputs:
  oracle/libglide_oracle.so      -- this project's C++ restatement of the
                                    reference's discrete operator and solver
                                    sequencing (binary64 and binary32 entry
                                    points), OpenMP over rows, and of its
                                    enthalpy column solver (binary64).
  oracle/_ref/libglide_ref32.so  -- the reference's own kernel sources
  oracle/_ref/libglide_ref64.so     (glide/cuda/*.cu) compiled as host C++ from
                                    the reference checkout and executed by the
                                    fiber emulator in simt_host.cpp; built only
                                    when the reference checkout is present.
  oracle/_ref/libglide_ref_gpu.so -- the same sources compiled unmodified for
                                    sm_100a with --use_fast_math (ref_gpu.cu),
                                    for timing the reference's kernels on the
                                    GPU (oracle/ref_gpu.py); built by nvcc when
                                    it and the reference checkout are present.

Usage: python oracle/build_oracle.py [--reference DIR] [--force]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
DEFAULT_REFERENCE = "/root/reference"

CXX = os.environ.get("GLIDE_CXX", "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++")
BASE_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              "-Wno-unused-variable", "-Wno-unused-but-set-variable"]


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources if s.exists())


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_oracle(force: bool = False) -> Path:
    out = HERE / "libglide_oracle.so"
    srcs = [HERE / "glide_oracle.cpp", HERE / "glide_oracle.hpp", HERE / "enthalpy_oracle.cpp"]
    if force or _stale(out, srcs):
        _run([CXX, *BASE_FLAGS, "-march=x86-64-v2", str(HERE / "glide_oracle.cpp"),
              str(HERE / "enthalpy_oracle.cpp"), "-o", str(out)])
    return out


# Constants the reference injects into its enthalpy kernels, in the order of
# glide/enthalpy.py:231-238; K_COLD and E_SCALE follow as expressions.
ENTHALPY_CONSTANTS = ["RHO_I", "RHO_W", "C_I", "K_I", "L_HEAT", "T_REF", "T_MELT", "BETA_CC", "GRAVITY",
                      "K_TEMP_FACTOR", "MASS_FLUX_REG", "MASS_FLUX_REG_YR"]


def enthalpy_defines(reference: str) -> str:
    """The #define block the reference prepends to enthalpy.cu
    (glide/enthalpy.py:229-246): each constant as a binary32 literal of its
    Python value.  The numeric module-level assignments of glide/enthalpy.py
    are evaluated in order, with no builtins."""
    src = (Path(reference) / "glide" / "enthalpy.py").read_text()
    ns: dict[str, float] = {}
    for line in src.splitlines():
        m = re.match(r"^([A-Z][A-Z0-9_]*)\s*=\s*([0-9A-Z_.+\-*/() e]+?)\s*(#.*)?$", line)
        if m:
            try:
                ns[m.group(1)] = float(eval(m.group(2), {"__builtins__": {}}, dict(ns)))
            except Exception:
                pass
    missing = [k for k in ENTHALPY_CONSTANTS if k not in ns]
    if missing:
        raise RuntimeError(f"constants not found in glide/enthalpy.py: {missing}")
    lines = [f"#define {k} {ns[k]}f" for k in ENTHALPY_CONSTANTS]
    lines += ["#define K_COLD (K_I/C_I)", "#define E_SCALE (C_I * (T_MELT - T_REF))"]
    return "\n".join(lines) + "\n"


def build_reference(reference: str, force: bool = False) -> list[Path]:
    cuda_dir = Path(reference) / "glide" / "cuda"
    if not cuda_dir.is_dir():
        print(f"reference kernels not found under {cuda_dir}; skipping oracle/_ref", flush=True)
        return []
    REF_OUT.mkdir(exist_ok=True)
    defines = REF_OUT / "enthalpy_defines.h"
    text = enthalpy_defines(reference)
    if not defines.exists() or defines.read_text() != text:
        defines.write_text(text)
    srcs = [HERE / "ref_harness.cpp", HERE / "simt_host.cpp", HERE / "simt_host.hpp", defines,
            *sorted(cuda_dir.glob("*.cu"))]
    outs = []
    for bits, defs in ((32, []), (64, ["-DGLIDE_REF_FP64"])):
        out = REF_OUT / f"libglide_ref{bits}.so"
        if force or _stale(out, srcs):
            _run([CXX, *BASE_FLAGS, "-w", f"-I{cuda_dir}", f"-I{HERE}", f"-I{REF_OUT}", *defs,
                  str(HERE / "ref_harness.cpp"), str(HERE / "simt_host.cpp"), "-o", str(out)])
        outs.append(out)
    nvcc = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    if Path(nvcc).exists():
        out = REF_OUT / "libglide_ref_gpu.so"
        gsrcs = [HERE / "ref_gpu.cu", *sorted(cuda_dir.glob("*.cu"))]
        if force or _stale(out, gsrcs):
            _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--use_fast_math",
                  "-Xcompiler", "-fPIC", "-shared", "-w", f"-I{cuda_dir}", str(HERE / "ref_gpu.cu"), "-o",
                  str(out), "-lcudart"])
        outs.append(out)
    return outs


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GLIDE_REFERENCE", DEFAULT_REFERENCE))
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--skip-oracle", action="store_true")
    args = ap.parse_args(argv)
    if not args.skip_oracle and (HERE / "glide_oracle.cpp").exists():
        build_oracle(args.force)
    build_reference(args.reference, args.force)
    return 0


if __name__ == "__main__":
    sys.exit(main())
