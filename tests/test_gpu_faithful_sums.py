"""Parity against the reference's own summation order.

press.f95 forms rhsav (with the volume), the SOR residual and pav as serial
FP32 loops (press.f95:66-75, 87-99, 123-133).  The library's default sums
are exact (order-free) instead; its reference-order mode
(les_ctx_set_reduction_mode, LES_RED_F_* bits) restates the serial loops.
Here the CUDA path in that mode is compared bit for bit with the oracle in
its faithful mode (ORACLE_RED_F_*, the same bits), one sum at a time and all
three together, and over the reference's 200 steps of the 150 x 150 x 90
benchmark case.  The tolerance stated for the physics fields, 1e-5 relative
L2 on u, v, w, p against the reference's algorithm, is asserted beside the
bit-exact check.
"""
import numpy as np
import pytest

import oracle
from les_halo_b200 import GpuLes, abi, fields as FL, synthetic_case
from tests.helpers import assert_bitexact, rel_l2

pytestmark = pytest.mark.gpu
TOL_REL_L2 = 1e-5
ALL = FL.STATE + FL.MASKS


def _pair(ip, jp, kp, seed, **kw):
    case = synthetic_case(ip, jp, kp, seed=seed, masks_and_poisson=oracle.masks_and_poisson, **kw)
    return case, case.copy()


def _compare(gpu, ref_case, names=ALL):
    got = gpu.download(names)
    want = {n: ref_case.a(n) for n in names}
    for n in ("u", "v", "w", "p"):
        assert rel_l2(got[n], want[n]) <= TOL_REL_L2, n
    assert_bitexact(got, want, ref_case.ip, ref_case.jp, ref_case.kp, names)
    return got


@pytest.fixture
def oracle_mode():
    yield oracle.set_reduction_mode
    oracle.set_reduction_mode(oracle.RED_CANONICAL)


@pytest.mark.parametrize("mode", [abi.LES_RED_F_RHSAV, abi.LES_RED_F_SOR, abi.LES_RED_F_PAV,
                                  abi.LES_RED_FAITHFUL])
@pytest.mark.parametrize("dims", [(24, 20, 16), (33, 19, 12), (40, 8, 7)])
def test_reference_order_sums_bitexact(require_gpu, oracle_mode, mode, dims):
    # odd ip and jp included: the residual's colour walk and the
    # per-colour SOR path (odd jp) take other branches there
    assert (abi.LES_RED_F_RHSAV, abi.LES_RED_F_SOR, abi.LES_RED_F_PAV) == \
        (oracle.RED_F_RHSAV, oracle.RED_F_SOR, oracle.RED_F_PAV)
    ip, jp, kp = dims
    oracle_mode(mode)
    ref, dev = _pair(ip, jp, kp, seed=ip * 5 + jp)
    gpu = GpuLes(dev)
    gpu.set_reduction_mode(mode)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    for n in range(1, 5):
        iters = oracle.run_steps(ref, n, 1)
        gpu.step(n, 1)
        assert gpu.metrics()["sor_iters"] == iters[0]
        _compare(gpu, ref)
    gpu.close()


def test_reference_order_residual_stops_early(require_gpu, oracle_mode):
    # a threshold the FP32 serial residual crosses part-way through the
    # iterations: the stop decision and the iteration count follow it
    ip, jp, kp = 20, 16, 10
    oracle_mode(oracle.RED_FAITHFUL)
    ref, dev = _pair(ip, jp, kp, seed=4)
    for c in (ref, dev):
        c.params.pjuge = 6.0e3
        c.params.nmaxp = 25
    gpu = GpuLes(dev)
    gpu.set_reduction_mode(abi.LES_RED_FAITHFUL)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    for n in range(1, 4):
        iters = oracle.run_steps(ref, n, 1)
        gpu.step(n, 1)
        m = gpu.metrics()
        assert m["sor_iters"] == iters[0] < 25
        _compare(gpu, ref)
    gpu.close()


def test_mode_switch_back_to_exact_sums(require_gpu):
    # the mode is per context and captured steps follow a switch: after
    # faithful steps, exact-sum steps equal those of a context that never
    # left the default (given the same state)
    ip, jp, kp = 24, 20, 16
    _, a = _pair(ip, jp, kp, seed=8)
    g1 = GpuLes(a)
    g1.set_reduction_mode(abi.LES_RED_FAITHFUL)
    g1.warmup(1)
    g1.step(1, 2)
    mid = g1.download(FL.STATE)
    b = a.copy()
    for n in FL.STATE:
        b.arrays[n] = mid[n].copy(order="F")
    g1.set_reduction_mode(abi.LES_RED_CANONICAL)
    g1.step(3, 2)
    g2 = GpuLes(b)
    g2.step(3, 2)
    assert_bitexact(g1.download(ALL), g2.download(ALL), ip, jp, kp, ALL)
    g1.close()
    g2.close()


def test_reference_order_sums_refuse_refined_press(require_gpu):
    _, a = _pair(24, 20, 16, seed=2)
    g = GpuLes(a)
    g.set_reduction_mode(abi.LES_RED_F_PAV)
    with pytest.raises(abi.LesError):
        g.press_refine_fp64(1, 0, 1e-9)
    g.set_reduction_mode(abi.LES_RED_CANONICAL)
    g.press_refine_fp64(1, 0, 1e-9)
    with pytest.raises(abi.LesError):
        g.set_reduction_mode(abi.LES_RED_FAITHFUL)
    with pytest.raises(abi.LesError):
        abi.check(abi.lib().les_ctx_set_reduction_mode(g.ctx, 8))
    g.close()


@pytest.mark.slow
def test_benchmark_case_200_steps_reference_order(require_gpu, oracle_mode):
    # the 150 x 150 x 90 benchmark case over the reference's 200 steps with
    # every global sum in the reference's serial FP32 order: bit-exact
    # against the oracle's faithful restatement on every state array.  The
    # same run with the default exact sums (bit-exact against the oracle's
    # canonical mode in test_gpu_step.py) is then compared field by field
    # to report the effect of the summation order alone.
    ip, jp, kp = 150, 150, 90
    oracle_mode(oracle.RED_FAITHFUL)
    ref, dev = _pair(ip, jp, kp, seed=1)
    canon = dev.copy()
    gpu = GpuLes(dev)
    gpu.set_reduction_mode(abi.LES_RED_FAITHFUL)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    oracle.run_steps(ref, 1, 200)
    gpu.step(1, 200)
    assert gpu.metrics()["n"] == 200
    faithful = _compare(gpu, ref)
    gpu.close()
    gc = GpuLes(canon)
    gc.warmup(1)
    gc.step(1, 200)
    exact = gc.download(FL.STATE)
    gc.close()
    gap = {n: rel_l2(exact[n], faithful[n]) for n in ("u", "v", "w", "p")}
    print("exact-sum vs reference-order sums after 200 steps, relative L2:",
          " ".join(f"{n}={v:.2e}" for n, v in gap.items()))
    # the order of the sums alone moves the turbulent trajectory by O(1e-6)
    # on the velocities and O(1e-5) on p over 200 steps
    for n in ("u", "v", "w"):
        assert gap[n] < 1e-5, (n, gap)
    assert gap["p"] < 1e-4, gap
