"""Ranks as separate processes sharing one GPU, over gloo (the NCCL paths
need a GPU per rank): the x-decomposed domain with DistExchange staging its
halo blocks and sums through host memory, and the sharded ensemble of
bench.py.  Each process has its own context; no kernel waits on another
process (every exchange is a host-side send/recv), so sharing the GPU is
safe."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold", "rhs", "sm"]
IP, JP, KP, NSTEPS = 100, 40, 30, 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, n, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=n, timeout=datetime.timedelta(seconds=120))
    return dist


def _dd_rank(rank, n, port, q):
    dist = _init(rank, n, port)
    r = None
    try:
        from les_halo_b200 import synthetic_case, fields as FL
        from les_halo_b200 import decomp as D
        case = synthetic_case(IP, JP, KP, seed=5, dt=0.05, nmaxp=50)
        slab = D.split_columns(IP, n, 16)[rank]
        r = D.DDRank(case, slab)
        parts = [None] * n
        dist.all_gather_object(parts, r.area_part())
        r.set_owned(sum(parts))
        D.run_steps([r], D.DistExchange(r, dist, device="cpu"), 1, NSTEPS, case.params.nmaxp, case.params.ical)
        r.gpu.sync()
        loc = r.gpu.download(NAMES)
        out = {}
        for nm in NAMES:
            (llo, lhi) = FL.bounds(nm, slab.im, JP, KP)[0]
            a = slab.olo if slab.west is not None else llo
            b = slab.ohi if slab.east is not None else lhi
            out[nm] = (a + slab.off, loc[nm][a - llo:b - llo + 1].copy())
        q.put((rank, out, r.gpu.metrics()))
        dist.barrier()
    finally:
        if r is not None:
            r.close()
        dist.destroy_process_group()


def _spawn(target, n, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, n, port, q) + args) for r in range(n)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(n)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return sorted(res, key=lambda x: x[0])


def test_decomposed_domain_two_processes(require_gpu):
    from les_halo_b200 import GpuLes, synthetic_case, fields as FL
    case = synthetic_case(IP, JP, KP, seed=5, dt=0.05, nmaxp=50)
    g = GpuLes(case)
    try:
        g.step(1, NSTEPS)
        g.sync()
        want, wm = g.download(NAMES), g.metrics()
    finally:
        g.close()
    res = _spawn(_dd_rank, 2)
    for nm in NAMES:
        got = FL.alloc(nm, IP, JP, KP)
        glo = FL.bounds(nm, IP, JP, KP)[0][0]
        for _, out, _ in res:
            i0, blk = out[nm]
            got[i0 - glo:i0 - glo + blk.shape[0]] = blk
        assert np.array_equal(got.view(np.uint32), want[nm].view(np.uint32)), nm
    for _, _, m in res:
        assert (m["sor_iters"], m["rhsav"], m["pav"]) == (wm["sor_iters"], wm["rhsav"], wm["pav"])


def _ens_rank(rank, n, port, q):
    dist = _init(rank, n, port)
    try:
        import bench
        bench.ENSEMBLE.update(members=6, size_lo=32, size_hi=48, kp=24, steps=3, seq_steps=2)
        q.put((rank, bench.ensemble_bench(3, 3, n, rank, dist)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_two_processes(require_gpu):
    import bench
    saved = dict(bench.ENSEMBLE)
    try:
        bench.ENSEMBLE.update(members=6, size_lo=32, size_hi=48, kp=24, steps=3, seq_steps=2)
        doms = bench.ensemble_members()
    finally:
        bench.ENSEMBLE.clear()
        bench.ENSEMBLE.update(saved)
    cells = [ip * jp * 24 for ip, jp, _, _ in doms]
    res = _spawn(_ens_rank, 2)
    for _, out in res:
        assert "error" not in out, out
        assert out["ranks"] == 2 and out["cells"] == sum(cells) and out["members"] == 6
    assert res[0][1]["ensemble_ms_per_step"] == res[1][1]["ensemble_ms_per_step"]  # the slowest rank's
