"""The replica path of bench.py over torch.distributed, on CPU with two gloo
ranks: max-over-ranks timing, whole-job rates, and the reference arm that
runs on rank 0 only (the other ranks exit without work)."""
import argparse
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # rank r took 10+r ms on the device and 1+2r s end to end
        q.put((rank, bench.job_rates(10.0 + rank, 1.0 + 2.0 * rank, 1000, 5, 3, 2, dist, "cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_rank_and_the_job_total():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    for r in range(2):
        ms, e2e, value, e2e_value = res[r]
        assert (ms, e2e) == (11.0, 3.0)
        assert value == pytest.approx(2 * 1000 * 5 / 0.011 / 1e6)
        assert e2e_value == pytest.approx(2 * 1000 * 3 / 3.0 / 1e6)


def test_reference_arm_does_nothing_on_other_ranks(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(steps=1, warmup=3, gpus=2, impl="reference")
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""


def test_ensemble_shards_cover_every_member_once_and_balance():
    import bench
    cells = [ip * jp * 80 for ip, jp, _, _ in bench.ensemble_members()]
    assert len(cells) == 64 and bench.ensemble_members() == bench.ensemble_members()  # same on every rank
    for ws in (1, 2, 3, 4, 8):
        shards = bench.shard_members(cells, ws)
        assert sorted(m for s in shards for m in s) == list(range(64))
        loads = [sum(cells[m] for m in s) for s in shards]
        assert max(loads) - min(loads) <= max(cells)  # greedy bound
    # 5 -> r0, 4 -> r1, 2 -> r1 (4 < 5), 1 -> r0 (5 < 6)
    assert bench.shard_members([5, 1, 4, 2], 2) == [[0, 1], [2, 3]]


def _ens_rank_main(rank, port, q, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        failed = rank == fail_rank
        ms = float("inf") if failed else 20.0 + 5.0 * rank
        q.put((rank, bench.ensemble_job(ms, 1000 * (rank + 1), failed, dist, "cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fail_rank", [-1, 1])
def test_ensemble_job_takes_the_slowest_rank_and_all_cells(fail_rank):
    # a rank whose members failed still joins the collectives, so no rank hangs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_rank_main, args=(r, port, q, fail_rank)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    for r in range(2):
        ms, cells, failed = res[r]
        assert cells == 3000
        assert failed == (fail_rank >= 0)
        if fail_rank < 0:
            assert ms == 25.0
