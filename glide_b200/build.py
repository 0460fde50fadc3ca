"""Build the sm_100a C-ABI library in-tree: glide_b200/_lib/libglide_b200.so.

    python -m glide_b200.build [--force] [--verbose-ptxas]

nvcc cross-compiles for sm_100a without a GPU.  The library links only the
CUDA runtime; it exports the entry points declared in include/glide_b200.h.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libglide_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
UNITS = ["runtime.cu", "noalloc.cu", "enthalpy.cu", "io.cu"]
# Fast single-precision math (approximate division, square root, reciprocal
# cube root; flush-to-zero) for the binary32 smoother and tangent kernels, as
# the reference compiles its own kernels.  Binary64 code is unaffected.
EXTRA = os.environ.get("GLIDE_NVCC_EXTRA", "--use_fast_math").split()


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def sources() -> list[Path]:
    return (sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inc"))
            + sorted((ROOT / "include").glob("*.h")))


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources())


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not stale():
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", *EXTRA,
           "-Xcompiler", "-fPIC", "-shared", "-I", str(ROOT / "include"), "-I", str(CSRC),
           *[str(CSRC / f) for f in UNITS], "-o", str(LIB) + ".tmp", "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args(argv)
    build(a.force, a.verbose_ptxas)
    return 0


if __name__ == "__main__":
    sys.exit(main())
