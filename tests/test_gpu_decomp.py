"""The x-decomposed step on the GPU: 1, 2 and 3 ranks of one domain, all in
this process (LocalExchange: halo blocks and sums moved by device copies
ordered with CUDA events; no kernel waits on another), against the single
domain's les_step.  Every own cell, ghost and step scalar must be identical
bit for bit; with halos narrower than the momentum phases' reach the result
must differ (the check has teeth)."""
import numpy as np
import pytest

from les_halo_b200 import GpuLes, synthetic_case
from les_halo_b200 import decomp as D

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold", "rhs", "sm"]
IP, JP, KP, NSTEPS = 100, 40, 30, 3


@pytest.fixture(scope="module")
def single():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    case = synthetic_case(IP, JP, KP, seed=5, dt=0.05, nmaxp=50)
    g = GpuLes(case.copy())
    try:
        g.step(1, NSTEPS)
        g.sync()
        return case, g.download(NAMES), g.metrics()
    finally:
        g.close()


def _run(case, nranks, halo, sync_every):
    dd = D.DecomposedLes(case.copy(), nranks, halo=halo, sync_every=sync_every)
    try:
        dd.step(1, NSTEPS)
        dd.sync()
        return dd.download(NAMES), dd.metrics()
    finally:
        dd.close()


def _same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("nranks,halo,sync_every,sor", [(1, 16, 8, "passes"), (2, 16, 8, "passes"),
                                                        (3, 16, 8, "passes"), (2, 12, 6, "passes"),
                                                        (1, 16, 8, "colour"), (3, 16, 8, "colour"),
                                                        (2, 12, 6, "colour")])
def test_decomposed_step_is_the_single_domain_bit_for_bit(single, nranks, halo, sync_every, sor, monkeypatch):
    # passes: the one-iteration SOR pass kernels, partial sums finished on the
    # host side of the exchange; colour: the per-colour sweeps
    if sor == "colour":
        monkeypatch.setenv("LES_DD_SOR", "colour")
    case, want, wm = single
    got, ms = _run(case, nranks, halo, sync_every)
    bad = [n for n in NAMES if not _same(got[n], want[n])]
    assert not bad, bad
    for m in ms:  # every rank holds the global scalars of the last step
        for k in ("n", "sor_iters", "rhsav", "pav"):
            assert m[k] == wm[k], (k, m[k], wm[k])
    assert ms[-1]["uout"] == wm["uout"]  # the east rank holds the outflow face


def test_narrow_halo_is_not_exact(single):
    case, want, _ = single
    got, _ = _run(case, 2, 2, 1)
    assert any(not _same(got[n], want[n]) for n in ("u", "v", "w", "p"))


def test_nccl_transport_one_rank(single):
    """DistExchange over an NCCL group of one rank: the all-reduces of the
    sums go through NCCL on the context's stream (the halo exchange of a
    one-rank group is empty)."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    case, want, wm = single
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    r = None
    try:
        torch.cuda.set_device(0)
        slab = D.split_columns(IP, 1, 0)[0]
        r = D.DDRank(case.copy(), slab)
        r.set_owned(r.area_part())
        ex = D.DistExchange(r, dist, device="cuda")
        D.run_steps([r], ex, 1, NSTEPS, nmaxp=case.params.nmaxp, ical=case.params.ical)
        r.gpu.sync()
        got = r.gpu.download(NAMES)
        assert all(_same(got[n], want[n]) for n in NAMES)
        assert r.gpu.metrics()["pav"] == wm["pav"]
    finally:
        if r is not None:
            r.close()
        dist.destroy_process_group()
