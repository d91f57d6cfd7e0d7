"""A workload over every device entry of the library, for the bounds-checked
build: run as a child process (``python -m tests.checked_workload``) with
LES_B200_CHECKED=1 it loads liblesb200_checked.so, where every box index is
checked against its allocation, and prints one JSON line with the number of
out-of-range indices seen (les_bounds_violations) and a digest of every
deterministic result.  Without the variable it runs the plain library, so
the two can be compared: the checks must not change a single bit.  The step
adjoint accumulates with atomics (its sums are order-dependent), so it
reports norms instead of a digest.

Not collected by pytest (test_gpu_checked.py drives it).
"""
import ctypes as C
import hashlib
import json

import numpy as np

from les_halo_b200 import (Ensemble, GpuAdjoint, GpuLes, abi, fields as FL, set_drag, synthetic_case,
                           tke_gradient)

ALL = FL.STATE + FL.MASKS


def _digest(h, arrays):
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())


def main():
    L = abi.lib()
    out = {"lib": abi.LIB_PATH.name}
    h = hashlib.sha256()
    # time steps over ragged shapes, both sum modes
    for dims, mode in (((24, 20, 16), abi.LES_RED_CANONICAL), ((33, 19, 12), abi.LES_RED_FAITHFUL),
                       ((40, 8, 7), abi.LES_RED_CANONICAL), ((64, 48, 20), abi.LES_RED_CANONICAL)):
        case = synthetic_case(*dims, seed=sum(dims))
        gpu = GpuLes(case)
        gpu.set_reduction_mode(mode)
        gpu.warmup(1)
        gpu.step(1, 4)
        F = gpu.download(ALL)
        _digest(h, [F[n] for n in ALL])
        # the context's halo entries, read then written back
        for hid in range(len(abi.HALO_IDS)):
            buf = np.zeros(int(L.les_ctx_halo_floats(gpu.ctx, hid)), np.float32)
            abi.check(L.les_ctx_halo_read(gpu.ctx, hid, buf.ctypes.data))
            abi.check(L.les_ctx_halo_write(gpu.ctx, hid, buf.ctypes.data))
            _digest(h, [buf])
        gpu.close()
    out["steps"], h = h.hexdigest(), hashlib.sha256()
    # FP64-refined press: the iterative and the spectral correction
    for outer, inner in ((2, 10), (2, 0)):
        gpu = GpuLes(synthetic_case(24, 20, 12, seed=7))
        gpu.warmup(1)
        gpu.step(1, 1)
        gpu.press_refine_fp64(outer, inner, 0.0)
        gpu.step(2, 1)
        _digest(h, [gpu.download(["p"])["p"]])
        gpu.close()
    out["refine"] = h.hexdigest()
    # the step adjoint with a drag scale, over checkpoints
    case = synthetic_case(24, 20, 12, seed=3)
    case.params.nmaxp = 3
    gpu = GpuLes(case)
    gpu.warmup(1)
    set_drag(gpu, np.full((24, 20), 1.1, np.float32))
    adj = GpuAdjoint(gpu, 4, 3)
    J, g = tke_gradient(gpu, adj, 1, 4, ((2, 20), (2, 18), (1, 8)), 2)
    out["adjoint"] = {"J": J, **{k: float(np.linalg.norm(g[k])) for k in ("wp", "drag")},
                      "state": float(np.sqrt(sum(np.sum(g["state"][n].astype(np.float64) ** 2)
                                                 for n in FL.STATE)))}
    adj.close()
    gpu.close()
    # an ensemble of uneven domains
    members = [GpuLes(synthetic_case(*d, seed=s)) for d, s in (((24, 20, 16), 1), ((33, 19, 12), 2))]
    for m in members:
        m.warmup(1)
    h = hashlib.sha256()
    ens = Ensemble(members)
    ens.step(1, 3)
    ens.sync()
    for m in members:
        F = m.download(ALL)
        _digest(h, [F[n] for n in ALL])
    ens.close()
    for m in members:
        m.close()
    count = C.c_ulonglong(0)
    first = (C.c_int * 3)()
    st = L.les_bounds_violations(C.byref(count), first)
    out.update(ensemble=h.hexdigest(), status=int(st), violations=int(count.value), first=list(first))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
