"""Build recipe for the CPU oracle (test infrastructure only).

Outputs:
  oracle/libglide_oracle.so      -- this project's C++ restatement of the
                                    reference's discrete operator and solver
                                    sequencing (binary64 and binary32 entry
                                    points), OpenMP over rows.
  oracle/_ref/libglide_ref32.so  -- the reference's own kernel sources
  oracle/_ref/libglide_ref64.so     (glide/cuda/*.cu) compiled as host C++ from
                                    the reference checkout and executed by the
                                    fiber emulator in simt_host.cpp; built only
                                    when the reference checkout is present.

Usage: python oracle/build_oracle.py [--reference DIR] [--force]
"""
from __future__ import annotations

import argparse
import os
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
    srcs = [HERE / "glide_oracle.cpp", HERE / "glide_oracle.hpp"]
    if force or _stale(out, srcs):
        _run([CXX, *BASE_FLAGS, "-march=x86-64-v2", str(HERE / "glide_oracle.cpp"),
              "-o", str(out)])
    return out


def build_reference(reference: str, force: bool = False) -> list[Path]:
    cuda_dir = Path(reference) / "glide" / "cuda"
    if not cuda_dir.is_dir():
        print(f"reference kernels not found under {cuda_dir}; skipping oracle/_ref", flush=True)
        return []
    REF_OUT.mkdir(exist_ok=True)
    srcs = [HERE / "ref_harness.cpp", HERE / "simt_host.cpp", HERE / "simt_host.hpp",
            *sorted(cuda_dir.glob("*.cu"))]
    outs = []
    for bits, defs in ((32, []), (64, ["-DGLIDE_REF_FP64"])):
        out = REF_OUT / f"libglide_ref{bits}.so"
        if force or _stale(out, srcs):
            _run([CXX, *BASE_FLAGS, "-w", f"-I{cuda_dir}", f"-I{HERE}", *defs,
                  str(HERE / "ref_harness.cpp"), str(HERE / "simt_host.cpp"), "-o", str(out)])
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
