"""Batched ensemble: uneven domains advanced by one graph launch per step
must give, member by member, exactly what les_step gives on its own."""
import numpy as np
import pytest

import oracle
from les_halo_b200 import Ensemble, GpuLes, fields as FL, synthetic_case
from tests.helpers import assert_bitexact

pytestmark = pytest.mark.gpu
ALL = FL.STATE + FL.MASKS
# uneven sizes; (17, 15, 9) has odd jp, so that member takes the per-colour SOR path
DOMAINS = [((24, 20, 12), 3, 0.3), ((40, 26, 16), 4, 0.45), ((17, 15, 9), 5, 0.2), ((33, 18, 10), 6, 0.35)]


def _case(dims, seed, ustar):
    ip, jp, kp = dims
    return synthetic_case(ip, jp, kp, seed=seed, ustar=ustar, masks_and_poisson=oracle.masks_and_poisson)


def test_ensemble_equals_member_steps(require_gpu):
    cases = [_case(*d) for d in DOMAINS]
    solo = [GpuLes(c.copy()) for c in cases]
    members = [GpuLes(c.copy()) for c in cases]
    for g in solo + members:
        g.warmup(1)
    ens = Ensemble(members)
    ens.step(1, 4)  # includes the n == 1 broadcast step
    for g in solo:
        g.step(1, 4)
    l1 = ens.launches()
    assert l1 > 0
    ti = ens.tune_info()  # the ensemble autotuner ran once, at the first step
    assert len(ti["candidates"]) == 10 and ti["chosen"] in ti["candidates"]
    assert all(v > 0 for v in ti["candidates"].values())
    for (dims, _, _), a, b in zip(DOMAINS, members, solo):
        assert_bitexact(a.download(ALL), b.download(ALL), *dims, ALL)
        ma, mb = a.metrics(), b.metrics()
        assert ma == mb or all(np.float32(ma[k]).view(np.uint32) == np.float32(mb[k]).view(np.uint32)
                               for k in ma)
    # member calls after ensemble steps are ordered after them
    members[1].step(5, 1)
    solo[1].step(5, 1)
    ens.step(6, 2)
    for g in solo:
        g.step(6, 2)
    for (dims, _, _), a, b in zip(DOMAINS, members, solo):
        assert_bitexact(a.download(ALL), b.download(ALL), *dims, ALL)
    assert ens.launches() > l1
    ens.close()
    for g in solo + members:
        g.close()


def test_ensemble_member_against_oracle(require_gpu):
    # one member of an ensemble against the CPU oracle directly
    cases = [_case(*d) for d in DOMAINS[:2]]
    ref = cases[0].copy()
    members = [GpuLes(c) for c in cases]
    oracle.ifdata(ref, 1)
    for g in members:
        g.warmup(1)
    ens = Ensemble(members)
    ens.step(1, 3)
    oracle.run_steps(ref, 1, 3)
    dims = DOMAINS[0][0]
    assert_bitexact(members[0].download(ALL), {k: ref.a(k) for k in ALL}, *dims, ALL)
    ens.close()
    for g in members:
        g.close()


def test_ensemble_with_refined_members(require_gpu):
    # members on the FP64-refined press (spectral and SOR inner solves; the
    # refine tail is part of each member's captured step) give what they give
    # alone
    doms = [((24, 20, 12), 3, 0.3), ((40, 26, 16), 4, 0.45)]
    cases = [_case(*d) for d in doms]
    solo = [GpuLes(c.copy()) for c in cases]
    members = [GpuLes(c.copy()) for c in cases]
    for g, (outer, inner) in zip(solo + members, [(2, 0), (1, 6)] * 2):
        g.warmup(1)
        g.press_refine_fp64(outer, inner, 1e-9)
    ens = Ensemble(members)
    ens.step(1, 3)
    for g in solo:
        g.step(1, 3)
    for (dims, _, _), a, b in zip(doms, members, solo):
        assert_bitexact(a.download(ALL), b.download(ALL), *dims, ALL)
        assert a.refine_metrics() == b.refine_metrics()
    ens.close()
    for g in solo + members:
        g.close()
