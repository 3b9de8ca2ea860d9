"""Build libwt.so (the CUDA step library) in-tree with nvcc for sm_100a.

Usage: python -m windtunnel_b200.build [--force] [--verbose]

Each translation unit is compiled separately so that the exact-arithmetic
kernels can be built with --fmad=false while the float32 step keeps
multiply-add contraction. The shared object lands next to this file, where
windtunnel_b200._lib loads it from.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libwt.so"
OBJ_DIR = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-I", str(INCLUDE),
]
# translation unit -> extra flags
UNITS = {
    "wt_kernels_fast.cu": [],
    "wt_kernels_exact.cu": ["--fmad=false"],
    "wt_api.cu": [],
    "wt_voxel.cu": ["--fmad=false"],
    "wt_view.cu": ["--fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put the CUDA toolkit on PATH")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every unit that changed and link libwt.so; returns its path."""
    OBJ_DIR.mkdir(exist_ok=True)
    nv = nvcc()
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "wt.h"]
    objs = []
    for unit, extra in UNITS.items():
        src = CSRC / unit
        obj = OBJ_DIR / (unit[:-3] + ".o")
        objs.append(obj)
        if force or ptxas_info or _stale(obj, [src] + headers):
            cmd = [nv, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nv, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))


if __name__ == "__main__":
    main()
