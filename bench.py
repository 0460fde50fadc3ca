"""Benchmark: coupled SSA momentum + mass-conservation time steps per second.

Workload (default): the large dome of the thermomechanical configuration --
2048 x 2048 cells, dx = 750 m, 7 levels, dt = 5 a, dome radius 1200 km,
Gaussian random bed, log-normal smoothed beta, smb lapse 2e-3 /m -- one step
= one FASCD solve to a relative residual of 1e-8 (binary64), followed by the
H_prev <- H update.  Inputs are synthetic (seeded) with those shapes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun every rank solves its own
replica of the step (the solve does not shard: one domain per GPU) and
`value` is the steps/s of all ranks together, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

METRIC = "SSA+mass coupled steps/s at 2048^2 to rel. residual 1e-8"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--levels", type=int, default=7)
    ap.add_argument("--dx", type=float, default=750.0)
    ap.add_argument("--radius", type=float, default=1200e3)
    ap.add_argument("--dt", type=float, default=5.0)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--inner", type=int, default=None, help="mixed: binary32 V-cycles per defect correction")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--max-vcycles", type=int, default=40)
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="step", choices=["step", "sweeps"],
                    help="sweeps: only N fine-level Vanka sweeps on the workload (profiling case)")
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--presolve", type=int, default=0, help="sweeps mode: V-cycles run before timing")
    ap.add_argument("--sweep-blocks", type=int, default=2, help="Vanka sweep blocks per SM (1 or 2)")
    ap.add_argument("--schedule", default=None,
                    help="pre,post,finest,coarsest sweeps of the FASCD V-cycle (default: the reference's 10,20,50,200)")
    ap.add_argument("--omega", type=float, default=None, help="Vanka omega (default 0.5)")
    ap.add_argument("--relax", type=float, default=None, help="local Newton step length (native mode only)")
    ap.add_argument("--native", action="store_true",
                    help="native mode: corrected v prolongation and the configured Newton relaxation")
    ap.add_argument("--quick", action="store_true", help="time the solve only (no e2e, roofline, CPU leg)")
    ap.add_argument("--method", default=None, choices=["fascd", "newton"],
                    help="forward solve: FASCD V-cycles, or FASCD then Newton with the tangent multigrid")
    ap.add_argument("--switch", type=int, default=None, help="newton: switch at rel. residual 10^-k")
    ap.add_argument("--tangent-vcycles", type=int, default=None)
    ap.add_argument("--tangent-schedule", default=None, help="pre,post,finest,coarsest of the tangent multigrid")
    ap.add_argument("--tangent-omega", type=float, default=None)
    return ap.parse_args()


def apply_solver_options(h, a):
    h.set_tuning(sweep_blocks_per_sm=a.sweep_blocks)
    if a.native:
        h.set_reference_quirks(False)
    if a.schedule:
        pre, post, fin, coarse = (int(x) for x in a.schedule.split(","))
        h.set_fas(False, pre_steps=pre, post_steps=post, finest_steps=fin, coarsest_steps=coarse)
    kw = {}
    if a.omega is not None:
        kw["omega"] = a.omega
    if a.relax is not None:
        kw["relaxation"] = a.relax
    if kw:
        h.set_vanka(False, -1, **kw)
    h.set_tuning(forward_method=a.method, newton_switch_exp10=a.switch, tangent_vcycles=a.tangent_vcycles)
    if a.tangent_schedule:
        pre, post, fin, coarse = (int(x) for x in a.tangent_schedule.split(","))
        h.set_fas(2, pre_steps=pre, post_steps=post, finest_steps=fin, coarsest_steps=coarse)
    if a.tangent_omega is not None:
        h.set_vanka(2, -1, omega=a.tangent_omega)


def run_sweeps(a):
    """Profiling case: the workload's finest level and N fused Vanka sweeps."""
    import torch

    from cases import dome
    from glide_b200.hierarchy import Hierarchy
    dtype = torch.float64 if a.precision == "fp64" else torch.float32
    f = dome(a.size, a.dx, a.radius, seed=0)
    levels = a.levels if a.presolve > 0 else 1
    h = Hierarchy(a.size, a.size, a.dx, levels, dtype=dtype)
    h.set_tuning(sweep_blocks_per_sm=a.sweep_blocks)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        h.set(k, 0, torch.as_tensor(f[k]), restrict_down=True)
    if a.presolve > 0:  # move to the near-converged regime of later V-cycles
        h.set_fas(False, maximum_vcycles=a.presolve, relative_tolerance=0.0, absolute_tolerance=0.0)
        h.forward(a.dt, 0)
    h.set_rhs(0, a.dt)
    out = {"mode": "sweeps", "size": a.size, "presolve_vcycles": a.presolve,
           "sweep_blocks_per_sm": a.sweep_blocks}
    for label, n in (("first", 1), ("next", a.sweeps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h.vanka_sweep(0, a.dt, n)
        e1.record()
        torch.cuda.synchronize()
        out[f"ms_per_sweep_{label}"] = e0.elapsed_time(e1) / n
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd[1:1] = ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def sweeps_per_vcycle(levels, pre=10, post=20, finest=50, coarsest=200):
    """Fine-level-equivalent Vanka sweeps of one V-cycle (level l costs 4^-l)."""
    s = pre + post + finest
    for l in range(1, levels - 1):
        s += (pre + post) * 4.0 ** (-l)
    s += coarsest * 4.0 ** (-(levels - 1))
    return s


# ------------------------------------------------------------------ our arm
def run_ours(a, rank, world):
    import torch
    import torch.distributed as dist

    from cases import dome
    from glide_b200.hierarchy import Hierarchy

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    dtype = torch.float32 if a.precision == "fp32" else torch.float64
    f = dome(a.size, a.dx, a.radius, seed=0)
    h = Hierarchy(a.size, a.size, a.dx, a.levels, precision=a.precision)
    if a.inner is not None:
        h.set_tuning(mixed_inner_vcycles=a.inner)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        h.set(k, 0, torch.as_tensor(f[k]), restrict_down=True)
    h.set_fas(False, maximum_vcycles=a.max_vcycles, relative_tolerance=a.rtol, absolute_tolerance=0.0)
    apply_solver_options(h, a)
    fas = h.get_fas(False)
    stream = torch.cuda.current_stream()

    def step():
        st = h.forward(a.dt, 0)
        h.view("H_prev", 0).copy_(h.view("H", 0))
        h.restrict("H_prev", 0)
        return st

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    gpu_uuid = None
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        gpu_uuid = None
    sampler = ClockSampler(gpu_uuid)
    sampler.start()
    time.sleep(0.3)
    l0 = h.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    stats = [step() for _ in range(a.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    launches = h.launch_count() - l0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / a.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms = float(t.item())
    vcyc = float(np.mean([s["vcycles"] for s in stats]))
    final_rel = float(np.max([s["final_norm"] / s["initial_norm"] for s in stats]))
    if a.quick:  # schedule exploration: the solve only
        return {"ms_per_step": ms, "vcycles_per_step": vcyc, "final_relative_residual": final_rel,
                "precision": a.precision, "method": a.method, "switch": a.switch,
                "schedule": a.schedule, "omega": a.omega, "relax": a.relax, "native": a.native,
                "tangent": [a.tangent_vcycles, a.tangent_schedule, a.tangent_omega]}, None

    # dominant kernel: the fused fine-level Vanka sweep, timed alone
    n_sw = 20
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h.vanka_sweep(0, a.dt, 2)
    s0.record(stream)
    h.vanka_sweep(0, a.dt, n_sw)
    s1.record(stream)
    torch.cuda.synchronize()
    sweep_ms = s0.elapsed_time(s1) / n_sw
    itemsize = 8 if dtype == torch.float64 else 4
    ncell = a.size * a.size
    bytes_per_sweep = 15 * ncell * itemsize
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_sweep / (sweep_ms * 1e-3) / 1e9

    # end to end through the public Python API with host buffers
    host = {k: torch.as_tensor(f[k]).to(dtype).pin_memory() for k in ("bed", "beta", "smb", "H_prev")}
    out_u = torch.empty(h.view("u", 0).shape, dtype=dtype).pin_memory()
    out_v = torch.empty(h.view("v", 0).shape, dtype=dtype).pin_memory()
    out_H = torch.empty(h.view("H", 0).shape, dtype=dtype).pin_memory()
    k_e2e = max(1, min(a.steps, 2))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(k_e2e):
        h.set("bed", 0, host["bed"].to(dev, non_blocking=True), restrict_down=True)
        h.set("beta", 0, host["beta"].to(dev, non_blocking=True), restrict_down=True)
        h.set("smb", 0, host["smb"].to(dev, non_blocking=True), restrict_down=True)
        hp = host["H_prev"].to(dev, non_blocking=True)
        h.set("H_prev", 0, hp, restrict_down=True)
        h.set("H", 0, hp, restrict_down=True)
        h.forward(a.dt, 0)
        out_u.copy_(h.view("u", 0), non_blocking=True)
        out_v.copy_(h.view("v", 0), non_blocking=True)
        out_H.copy_(h.view("H", 0), non_blocking=True)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = x0.elapsed_time(x1) / k_e2e
    te = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te.item())
    h2d = sum(v.numel() * itemsize for v in host.values())
    d2h = (out_u.numel() + out_v.numel() + out_H.numel()) * itemsize

    res = {
        "metric": METRIC,
        "value": world * 1000.0 / ms,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp64": "f64", "fp32": "f32", "mixed": "f64 residual / f32 smoother"}[a.precision],
        "data": "synthetic (seeded dome, Gaussian random bed, log-normal beta)",
        "config": {"workload": f"dome {a.size}x{a.size}, dx={a.dx:g} m, {a.levels} levels, dt={a.dt:g} a, "
                               f"FASCD to rel. residual {a.rtol:g} (max {a.max_vcycles} V-cycles)",
                   "grid": [a.size, a.size], "levels": a.levels, "dt_years": a.dt,
                   "relative_tolerance": a.rtol, "vcycles_per_step": vcyc,
                   "final_relative_residual": final_rel,
                   "parallelism": f"replicas x{world} (one domain per GPU)",
                   "l2": "inputs larger than L2 (state + parameters ~0.5 GB per level-0 pass)"},
        "gpu_launches": int(launches),
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": "k_vanka_sweep (fine level)", "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "launch_ms": sweep_ms,
                     "algorithmic_bytes_per_launch": bytes_per_sweep},
        "clocks": clocks,
    }
    res["config"]["schedule"] = {k: fas[k] for k in ("pre_steps", "post_steps", "finest_steps", "coarsest_steps")}
    res["config"]["reference_quirks"] = not a.native
    spv = sweeps_per_vcycle(a.levels, fas["pre_steps"], fas["post_steps"], fas["finest_steps"],
                            fas["coarsest_steps"])
    return res, spv * vcyc


# -------------------------------------------------------------- CPU legs
def cpu_oracle_sample(a, sweeps_per_step, budget_s):
    """binary64 C++/OpenMP oracle: timed fine-level Vanka sweeps on the same
    workload, scaled to steps/s with the step's fine-sweep equivalents."""
    from cases import dome
    from oracle.glide_oracle import OracleHierarchy
    f = dome(a.size, a.dx, a.radius, seed=0)
    o = OracleHierarchy(a.size, a.size, a.dx, 1)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        o.set_field(k, f[k])
    lev = o.levels[0]
    lev.f_H[...] = lev.H_prev / a.dt + lev.smb
    n, t0 = 0, time.perf_counter()
    while True:
        lev.vanka_sweep(a.dt, 1)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= 50:
            break
    per_sweep = el / n
    cores = len(os.sched_getaffinity(0))
    return {"value": 1.0 / (per_sweep * sweeps_per_step), "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{n} fine-level Vanka sweeps of the binary64 oracle at {a.size}^2 "
                      f"({per_sweep:.3f} s each), scaled by {sweeps_per_step:.1f} fine-sweep equivalents per step"}


# V-cycles per step to 1e-8 of this workload, measured by the binary64 GPU
# solver; the CPU reference leg cannot run a 2048^2 step to convergence.
REF_VCYCLES_PER_STEP = 40.0


def run_reference(a):
    """The reference's own kernels (oracle/_ref, host build of its CUDA
    sources) with its host loop: compute_grounded, vanka_smooth, omega axpys."""
    import ctypes

    from cases import dome
    from oracle.refpy import RefKernels
    lib_path = ROOT / "oracle" / "_ref" / "libglide_ref32.so"
    if not lib_path.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/libglide_ref32.so was not built "
                                                    "(reference checkout absent at build time)"}
    k = RefKernels(fp64=False)
    f = dome(a.size, a.dx, a.radius, seed=0)
    n = a.size
    z = lambda *s: np.zeros(s, np.float32)
    u, v, H = z(n, n + 1), z(n + 1, n), f["H"].astype(np.float32)
    phi, mask = z(n, n), z(n, n)
    fu, fv = z(n, n + 1), z(n + 1, n)
    fH = (f["H_prev"] / a.dt + f["smb"]).astype(np.float32)
    bed, B, beta = (f[x].astype(np.float32) for x in ("bed", "B", "beta"))
    gamma = np.full((n, n), 0.1, np.float32)
    du, dv, dH = z(n, n + 1), z(n + 1, n), z(n, n)
    grid = (n // 14 + 1, n // 14 + 1)
    phys = (3.0, 1e-6, 0.1, 1.0, 1.0, 1e-5, 0.1, 0.0, 0.1, a.dx, a.dt)
    spv = sweeps_per_vcycle(a.levels)
    steps_t = []
    cores = len(os.sched_getaffinity(0))
    for _ in range(max(1, a.steps)):
        nsw, t0 = 0, time.perf_counter()
        while True:
            k.launch("compute_grounded", grid, (16, 16), (phi, H, bed, 0.1, 0.0, n, n, 14, 1))
            du.fill(0); dv.fill(0); dH.fill(0)
            k.launch("vanka_smooth", grid, (16, 16),
                     (du, dv, dH, mask, u, v, H, phi, fu, fv, fH, bed, B, beta, gamma, *phys,
                      n, n, 14, 1, 30, 0.5, 0.01, 1.0))
            u += np.float32(0.5) * du
            v += np.float32(0.5) * dv
            H += np.float32(0.5) * dH
            nsw += 1
            el = time.perf_counter() - t0
            if el > a.cpu_seconds / max(1, a.steps) or nsw >= 20:
                break
        steps_t.append(el / nsw * spv * REF_VCYCLES_PER_STEP)
    step_s = float(np.median(steps_t))
    val = 1.0 / step_s
    return {
        "metric": METRIC, "value": val, "unit": "steps/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dome)", "impl": "reference",
        "config": {"workload": f"dome {a.size}x{a.size}, dx={a.dx:g} m, {a.levels} levels, dt={a.dt:g} a",
                   "vcycles_per_step_assumed": REF_VCYCLES_PER_STEP},
        "cpu_baseline": {"value": val, "unit": "steps/s", "cores": cores, "kind": "reference",
                         "sample": f"reference vanka_smooth sweeps (host build of glide/cuda/*.cu, binary32) at "
                                   f"{n}^2, per-step work = {REF_VCYCLES_PER_STEP:g} V-cycles x {spv:.1f} "
                                   f"fine-sweep equivalents"},
        "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if a.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(a)), flush=True)
        return 0
    import torch
    import torch.distributed as dist
    if a.mode == "sweeps":
        run_sweeps(a)
        return 0
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    res, sweeps_per_step = run_ours(a, rank, world)
    if rank == 0 and world == 1 and not a.no_cpu_baseline and not a.quick:
        res["cpu_baseline"] = cpu_oracle_sample(a, sweeps_per_step, a.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
