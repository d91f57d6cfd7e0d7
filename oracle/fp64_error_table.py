"""Relative L2 error of the FP32 time step against the FP64 oracle, per field.

TEST INFRASTRUCTURE (run by hand; prints a table): the FP32 oracle is
bit-identical to the CUDA path (tests/test_gpu_step.py), so its distance to
the same algorithm in double precision (oracle/fp64.py) is the CUDA path's.

    python oracle/fp64_error_table.py 150 150 90 200
"""
import pathlib
import sys

import numpy as np

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1]))
import oracle  # noqa: E402
from oracle import fp64  # noqa: E402
from les_halo_b200 import fields as FL, synthetic_case  # noqa: E402

FIELDS = ["u", "v", "w", "p", "f", "g", "h", "usum", "vsum", "wsum", "sm"]


def errors(ip, jp, kp, steps, seed=1, refine=None):
    c32 = synthetic_case(ip, jp, kp, seed=seed, masks_and_poisson=oracle.masks_and_poisson)
    c64 = fp64.Case64(c32)
    oracle.ifdata(c32, 1)
    c64.ifdata(1)
    if refine:
        oracle.set_press_refine(*refine)
        fp64.lib().oracle_set_press_refine.argtypes = [oracle.C.c_int, oracle.C.c_int, oracle.C.c_double]
        fp64.lib().oracle_set_press_refine(*refine)
    try:
        for n in range(1, steps + 1):
            oracle.run_steps(c32, n, 1)
            c64.run_steps(n, 1)
    finally:
        oracle.set_press_refine(0, 0, 0.0)
        if refine:
            fp64.lib().oracle_set_press_refine(0, 0, 0.0)
    out = {}
    for n in FIELDS:
        a = FL.interior(n, c32.a(n), ip, jp, kp).astype(np.float64)
        b = FL.interior(n, c64.a(n), ip, jp, kp)
        out[n] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return out


if __name__ == "__main__":
    ip, jp, kp, steps = (int(x) for x in sys.argv[1:5])
    for label, ref in (("plain", None), ("refined (spectral, 1 correction)", (1, 0, 0.0))):
        e = errors(ip, jp, kp, steps, refine=ref)
        print(f"{ip}x{jp}x{kp}, {steps} steps, {label}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()),
              flush=True)
