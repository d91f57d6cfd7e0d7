"""FP64-refined pressure solve (les_press_refine_fp64) against the oracle's
restatement of the same algorithm, with SOR inner sweeps and with the
spectral inner solve.

The plain FP32 sweeps and every pointwise FP64 expression are bit-identical
on both sides; the FP64 sums (residual norms, pav) are reduced in different
orders, so p (which carries pav) may differ in its last bit and the norms
and pav agree to ~1e-12 relative.  Everything else in the step is bit-exact.
"""
import numpy as np
import pytest

import oracle
from les_halo_b200 import GpuLes, fields as FL, synthetic_case
from tests.helpers import assert_bitexact

pytestmark = pytest.mark.gpu
NOT_P = [n for n in FL.STATE + FL.MASKS if n != "p"]


def _pair(ip, jp, kp, seed):
    case = synthetic_case(ip, jp, kp, seed=seed, masks_and_poisson=oracle.masks_and_poisson)
    return case, case.copy()


def _ulps(a, b):
    ai, bi = a.view(np.int32).astype(np.int64), b.view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7fffffff), ai)
    bi = np.where(bi < 0, -(bi & 0x7fffffff), bi)
    return int(np.max(np.abs(ai - bi)))


def _run(outer, inner, tol, dims=(24, 20, 12), seed=7):
    ip, jp, kp = dims
    ref, dev = _pair(ip, jp, kp, seed)
    gpu = GpuLes(dev)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    oracle.run_steps(ref, 1, 1)
    gpu.step(1, 1)
    gpu.press_refine_fp64(outer, inner, tol)
    oracle.set_press_refine(outer, inner, tol)
    try:
        oracle.run_steps(ref, 2, 1)
    finally:
        oracle.set_press_refine(0, 0, 0.0)
    gpu.step(2, 1)
    got = gpu.download(FL.STATE + FL.MASKS)
    return ref, gpu, got, oracle.last_refine(), gpu.refine_metrics()


@pytest.mark.parametrize("outer,inner", [(1, 10), (3, 20)])
def test_refined_press_matches_oracle(require_gpu, outer, inner):
    ref, gpu, got, want_m, m = _run(outer, inner, 0.0)
    ip, jp, kp = ref.ip, ref.jp, ref.kp
    assert_bitexact(got, {k: ref.a(k) for k in NOT_P}, ip, jp, kp, NOT_P)
    assert _ulps(got["p"], ref.a("p")) <= 1
    assert m["outer"] == want_m["outer"] == outer
    assert m["rhsav"] == want_m["rhsav"]  # both the exact fixed-point sum over the same area
    for k in ("pav", "rel_initial", "rel_final"):
        assert abs(m[k] - want_m[k]) <= 1e-10 * abs(want_m[k]) + 1e-300, k
    assert m["rel_final"] < m["rel_initial"]
    gpu.close()


def test_refined_press_stops_at_tolerance(require_gpu):
    # a tolerance above the first residual: no correction, p is the FP32
    # sweeps' result re-centred with the FP64 pav
    ref, gpu, got, want_m, m = _run(3, 10, 10.0)
    assert m["outer"] == want_m["outer"] == 0
    assert m["rel_final"] == m["rel_initial"]
    assert _ulps(got["p"], ref.a("p")) <= 1
    gpu.close()


def test_refine_rejects_odd_jp(require_gpu):
    from les_halo_b200 import abi
    case = synthetic_case(16, 15, 8, seed=2)
    g = GpuLes(case)
    st = abi.lib().les_press_refine_fp64(g.ctx, 2, 10, 0.0)
    assert st == abi.LES_ERR_DIMS
    st = abi.lib().les_press_refine_fp64(g.ctx, 2, 0, 0.0)  # spectral: even ip and jp
    assert st == abi.LES_ERR_DIMS
    g.close()


@pytest.mark.parametrize("outer", [1, 2])
def test_spectral_refined_press_matches_oracle(require_gpu, outer):
    # inner = 0: the FP64 spectral solve (FFT kernels on the GPU, direct sums in
    # the oracle) solves the FP64 system in one correction; both agree to
    # FP64 rounding, so p after its FP32 rounding differs by at most an ulp
    ref, gpu, got, want_m, m = _run(outer, 0, 0.0)
    ip, jp, kp = ref.ip, ref.jp, ref.kp
    assert_bitexact(got, {k: ref.a(k) for k in NOT_P}, ip, jp, kp, NOT_P)
    assert _ulps(got["p"], ref.a("p")) <= 1
    assert m["outer"] == want_m["outer"] == outer
    assert m["rel_final"] <= 1e-12 and want_m["rel_final"] <= 1e-12
    assert abs(m["rel_initial"] - want_m["rel_initial"]) <= 1e-10 * want_m["rel_initial"]
    assert abs(m["pav"] - want_m["pav"]) <= 1e-10 * abs(want_m["pav"])
    gpu.close()


def test_spectral_refine_stops_after_one_correction(require_gpu):
    # with a 1e-9 tolerance the second correction is skipped
    ref, gpu, got, want_m, m = _run(3, 0, 1e-9)
    assert m["outer"] == want_m["outer"] == 1
    assert m["rel_final"] <= 1e-9
    gpu.close()
