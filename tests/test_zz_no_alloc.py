"""les_press_rhs_noalloc: press.f95:49-81 on device arrays with no device
allocation, against the allocating per-routine entry les_press_.

The file name sorts last so the GPU test also runs after every other test
in one session (the static scratch must not depend on what ran before).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from les_halo_b200 import abi, fields as FL, synthetic_case
from tests.helpers import assert_bitexact

I = lambda x: C.byref(C.c_int(x))
Fv = lambda x: C.byref(C.c_float(x))
NAMES = ["rhs", "u", "dx1", "v", "dy1", "w", "dzn", "f", "g", "h", "cn1", "cn2l", "p", "cn2s",
         "cn3l", "cn3s", "cn4l", "cn4s"]
OUT = ["rhs", "f", "g", "h"]


def _press_inputs(ip, jp, kp, seed):
    case = synthetic_case(ip, jp, kp, seed=seed, masks_and_poisson=oracle.masks_and_poisson)
    oracle.ifdata(case, 1)
    oracle.run_steps(case, 1, 2)
    base = {n: case.a(n).copy(order="F") for n in NAMES}
    rhs = FL.alloc("rhs", ip, jp, kp)
    rhs[...] = np.random.default_rng(seed).standard_normal(rhs.shape).astype(np.float32)
    base["rhs"] = rhs  # garbage: elements press never writes must survive
    return case.params.dt, base


def _via_press_entry(ip, jp, kp, dt, base):
    """Existing entry point (host arrays, allocates its working set)."""
    b = {n: a.copy(order="F") for n, a in base.items()}
    args = [FL.ptr(b[n]) for n in NAMES]
    it = C.c_int()
    abi.check(abi.lib().les_press_(I(kp), I(jp), I(ip), *args[:10], Fv(dt), *args[10:], I(4), I(10),
                                   C.byref(it)))
    return {n: b[n] for n in OUT}


def _oracle_rhsav(ip, jp, kp, dt, base):
    L = oracle.lib()
    a = {n: x.copy(order="F") for n, x in base.items()}
    args = [FL.ptr(a[n]) for n in NAMES]
    out = C.c_float()
    fn = L.oracle_press
    i, f, p = C.c_int, C.c_float, C.c_void_p
    # the full signature: pointers must not go through ctypes' default int
    fn.argtypes = [i, i, i] + [p] * 10 + [f] + [p] * 8 + [i, i, p, p, p]
    fn.restype = C.c_int
    fn(kp, jp, ip, *args[:10], dt, *args[10:], 4, 10, None, C.byref(out), None)
    return out.value


def test_rejects_grids_beyond_the_static_scratch():
    # checked before any device work: runs without a GPU
    L = abi.lib()
    dummy = np.zeros(16, np.float32)
    ptrs = [dummy.ctypes.data] * 10
    st = L.les_press_rhs_noalloc(8, 4096, 4096, *ptrs, 0.1, None, None)
    assert st == abi.LES_ERR_DIMS
    assert "static scratch" in L.les_last_error_string().decode()
    st = L.les_press_rhs_noalloc(8, 8, 8, None, *ptrs[1:], 0.1, None, None)
    assert st == abi.LES_ERR_BAD_ARG


@pytest.mark.gpu
def test_two_calls_in_a_row_match_press_entry(require_gpu):
    import torch

    dev = torch.device("cuda:0")
    cases = [(40, 30, 20, 21), (21, 14, 11, 13)]  # different block counts on purpose
    prepared = []
    for ip, jp, kp, seed in cases:
        dt, base = _press_inputs(ip, jp, kp, seed)
        want = _via_press_entry(ip, jp, kp, dt, base)
        rhsav_want = _oracle_rhsav(ip, jp, kp, dt, base)
        d = {n: torch.from_numpy(np.asarray(base[n]).ravel(order="F").copy()).to(dev)
             for n in ["rhs", "u", "dx1", "v", "dy1", "w", "dzn", "f", "g", "h"]}
        d["rhsav"] = torch.full((1,), float("nan"), device=dev)
        prepared.append((ip, jp, kp, dt, base, want, rhsav_want, d))

    L = abi.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(ip, jp, kp, dt, d):
        p = lambda n: C.c_void_p(d[n].data_ptr())
        abi.check(L.les_press_rhs_noalloc(kp, jp, ip, p("rhs"), p("u"), p("dx1"), p("v"), p("dy1"),
                                          p("w"), p("dzn"), p("f"), p("g"), p("h"), dt, p("rhsav"),
                                          C.c_void_p(stream)))

    # a first call on a throw-away copy does the one-time scratch lookup
    ip, jp, kp, dt, _, _, _, d0 = prepared[1]
    call(ip, jp, kp, dt, {n: t.clone() for n, t in d0.items()})
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for ip, jp, kp, dt, _, _, _, d in prepared:
        call(ip, jp, kp, dt, d)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free_before

    for ip, jp, kp, dt, base, want, rhsav_want, d in prepared:
        got = {n: d[n].cpu().numpy().reshape(base[n].shape, order="F") for n in OUT}
        assert_bitexact(got, want, ip, jp, kp, OUT)
        assert np.float32(d["rhsav"].item()).view(np.uint32) == np.float32(rhsav_want).view(np.uint32)
