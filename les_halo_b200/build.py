"""Build liblesb200.so (sm_100a) in-tree with nvcc.

The library is compiled strict-IEEE (``--fmad=false``, IEEE division and
square root, no flush-to-zero) so that every kernel reproduces the
reference's single-precision expression order bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblesb200.so"
CHECKED = PKG / "liblesb200_checked.so"
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


def _run(cmd) -> str:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed: " + " ".join(cmd[-3:]))
    return res.stderr


def _compile_all(targets, verbose: bool) -> dict:
    """targets: {library path: extra nvcc flags}.  Every translation unit of
    every library compiles to an object concurrently (nvcc runs one source
    at a time), then each library links; returns {library: ptxas report}."""
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    jobs = []
    for out, extra in targets.items():
        for s in SOURCES:
            obj = objdir / f"{out.stem}.{Path(s).stem}.o"
            jobs.append((out, obj, [NVCC, *flags, *extra, "-I", str(ROOT / "include"), "-I", str(CSRC),
                                    "-c", "-o", str(obj), str(CSRC / s)]))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(lambda j: _run(j[2]), jobs))
    reports = {}
    for out in targets:
        objs = [str(j[1]) for j in jobs if j[0] == out]
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(out), *objs, "-ldl"])
        reports[out] = "".join(log for j, log in zip(jobs, logs) if j[0] == out)
        if verbose:
            sys.stderr.write(reports[out])
    return reports


def build(force: bool = False, verbose: bool = False, checked: bool = True) -> Path:
    """liblesb200.so, and (checked=True) liblesb200_checked.so: the same
    sources with LES_CHECKED, every box index checked against its
    allocation (les_bounds_violations)."""
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        list(CSRC.glob("*.inc")) + \
        list((ROOT / "include").glob("*.h")) + [Path(__file__)]
    targets = {}
    if force or _stale(LIB, deps):
        targets[LIB] = []
    if checked and (force or _stale(CHECKED, deps)):
        targets[CHECKED] = ["-DLES_CHECKED"]
    if targets:
        reports = _compile_all(targets, verbose)
        if LIB in reports:
            (PKG / "ptxas_info.txt").write_text(reports[LIB])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
