"""Build liblesb200.so (sm_100a) in-tree with nvcc.

The library is compiled strict-IEEE (``--fmad=false``, IEEE division and
square root, no flush-to-zero) so that every kernel reproduces the
reference's single-precision expression order bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblesb200.so"
SOURCES = ["les_lib.cu", "les_setup.cu", "les_noalloc.cu", "les_netcdf.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-Xptxas", "-v",
    "-shared",
]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        list(CSRC.glob("*.inc")) + \
        list((ROOT / "include").glob("*.h")) + [Path(__file__)]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-I", str(CSRC),
               "-o", str(LIB), *[str(CSRC / s) for s in SOURCES]]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode != 0:
            raise RuntimeError("nvcc failed for liblesb200.so")
        (PKG / "ptxas_info.txt").write_text(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
