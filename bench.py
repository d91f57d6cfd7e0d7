#!/usr/bin/env python
"""Benchmark of the B200 LES time step (one JSON line on rank 0).

Workload: the 600x600x120 plain FP32 step (synthetic terrain at 35% plan
area, heights to 120 m, log-law inflow with frozen noise, dt = 0.05 s, red-
black SOR with 50 sweeps per step).  One "step" is one full time step of
velnw, bondv1, velfg, feedbf, les, adam and press (main_ocl.f95:264-299).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank advances its own replica of the domain
(the single domain does not shard; replicas only) and `value` is the sum of
the ranks' throughput, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time-step Mpts/s: plain vs FP64-refined press at ≤1e-5 err; adjoint/fwd cost"
WORKLOAD = dict(ip=600, jp=600, kp=120, plan_area=0.35, h_max=120.0, dt=0.05, nmaxp=50, seed=1)
SOR_BYTES_PER_CELL_PER_ITER = 12.0   # algorithmic bytes of one SOR iteration: p read, rhs read, p write
STEP_BYTES_PER_CELL = 204.0 + 12.0 * 50  # algorithmic bytes per cell per step at 50 SOR iterations
# aveflow's running sums (aveflow.f95:72-88): read u, v, w, p, sm (20 B),
# read and write the ten sums (80 B)
AVE_BYTES_PER_CELL = 100.0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def job_rates(ms_total, e2e_s, cells, steps, e2e_steps, ws, dist=None, device="cpu"):
    """Max-over-ranks device and end-to-end times and the whole-job rates in
    Mpts/s: every rank advances its own replica of `cells` cells, so the job
    moves ws * cells per step in the slowest rank's time."""
    import torch
    t = torch.tensor([ms_total, e2e_s], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_total, e2e_s = float(t[0]), float(t[1])
    value = ws * cells * steps / (ms_total / 1e3) / 1e6
    e2e_val = ws * cells * e2e_steps / e2e_s / 1e6
    return ms_total, e2e_s, value, e2e_val


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_desc(ip, jp, kp):
    """The workload's name in both arms' config (identical strings)."""
    W = WORKLOAD
    return (f"LES plain FP32 step {ip}x{jp}x{kp} ({round(W['plan_area'] * 100)}% plan area, heights "
            f"<={W['h_max']:g} m, dt={W['dt']:g}, SOR {W['nmaxp']} sweeps/step)")


def native_libs():
    """Shared libraries of this repository mapped into the process."""
    out = set()
    try:
        for ln in Path("/proc/self/maps").read_text().splitlines():
            f = ln.split()[-1] if ln.split() else ""
            if f.endswith(".so") and f.startswith(str(ROOT)):
                out.add(str(Path(f).relative_to(ROOT)))
    except OSError:
        pass
    return sorted(out)


def make_case():
    """The workload built with the library's setup routines (masks and
    Poisson coefficients on the device)."""
    import les_halo_b200 as lh
    W = WORKLOAD
    return lh.synthetic_case(W["ip"], W["jp"], W["kp"], seed=W["seed"], dt=W["dt"], nmaxp=W["nmaxp"],
                             plan_area=W["plan_area"], h_max=W["h_max"])


def oracle_case():
    """The same workload built by the CPU oracle alone (no liblesb200.so)."""
    import oracle
    W = WORKLOAD
    return oracle.synthetic_case(W["ip"], W["jp"], W["kp"], seed=W["seed"], dt=W["dt"], nmaxp=W["nmaxp"],
                                 plan_area=W["plan_area"], h_max=W["h_max"])


def cpu_baseline(threads: int, steps=2):
    """The oracle (CPU restatement of the reference's Fortran step) on the
    workload itself: after the ifdata warm-up and one untimed step (the
    n == 1 inflow broadcast), `steps` full time steps, timed.  About 20 s of
    work on a 16-core host at 600 x 600 x 120."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle
    case = oracle_case()
    oracle.ifdata(case, 1)
    oracle.run_steps(case, 1, 1)  # untimed first step (n==1 broadcast)
    t0 = time.perf_counter()
    oracle.run_steps(case, 2, steps)
    dt = time.perf_counter() - t0
    cells = case.ip * case.jp * case.kp
    return {"value": round(cells * steps / dt / 1e6, 3), "unit": "Mpts/s", "cores": threads,
            "kind": "port",
            "sample": f"{steps} full time steps (n=2..{steps + 1}) of the {case.ip}x{case.jp}x{case.kp} "
                      f"workload itself, after the warm-up and one untimed step; oracle C++ restatement "
                      f"of the Fortran CPU path, OpenMP {threads} threads, {dt:.2f} s"}


def run_reference(args):
    """The reference's CPU time step on the host cores, on the same
    workload, metric and steps as the GPU arm: W untimed steps, then K
    timed full steps of the whole grid.  The reference's Fortran cannot be
    built here (no Fortran compiler), so its line-by-line C++ restatement
    (the oracle, OpenMP over all host threads) stands for it; the case is
    built by the oracle alone, so the library under test is never loaded."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle
    W = WORKLOAD
    case = oracle_case()
    ip, jp, kp = case.ip, case.jp, case.kp
    oracle.ifdata(case, 1)
    n = 1
    for _ in range(args.warmup):
        oracle.run_steps(case, n, 1)
        n += 1
    iters = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        iters += oracle.run_steps(case, n, 1)
        n += 1
    dt = time.perf_counter() - t0
    val = ip * jp * kp * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "Mpts/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded terrain + log-law inflow)",
        "config": {"workload": workload_desc(ip, jp, kp), "grid": [ip, jp, kp],
                   "sor_iters": int(max(iters)) if iters else W["nmaxp"],
                   "parallelism": f"host cores x{threads}", "l2": "CPU run"},
        "cpu_baseline": {"value": round(val, 3), "unit": "Mpts/s", "cores": threads, "kind": "port",
                         "sample": f"each step: one full time step of the {ip}x{jp}x{kp} workload; oracle "
                                   "C++ restatement of the reference Fortran (no Fortran compiler here to "
                                   f"build the reference itself), OpenMP {threads} threads"},
        "e2e": {"value": round(val, 3), "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "native_libs": native_libs(),
    }
    print(json.dumps(line), flush=True)
    return 0


REFINE = dict(outer=2, inner=0, tol=1e-9)  # inner 0: the FP64 spectral inner solve
ENSEMBLE = dict(members=64, size_lo=96, size_hi=256, kp=80, ustar_lo=0.2, ustar_hi=0.5, seed=2024, steps=200,
                seq_steps=20)


def ensemble_members():
    """The ensemble's domains, the same on every rank: (ip, jp, u*, seed)."""
    E = ENSEMBLE
    rng = np.random.default_rng(E["seed"])
    out = []
    for m in range(E["members"]):
        ip, jp = (int(x) for x in rng.integers(E["size_lo"], E["size_hi"] + 1, size=2))
        out.append((ip, jp, float(rng.uniform(E["ustar_lo"], E["ustar_hi"])), E["seed"] + 1 + m))
    return out


def shard_members(cells, ws):
    """Greedy balance of independent members over ws ranks: largest first,
    each onto the least-loaded rank (ties: lower rank).  Returns each rank's
    member indices in increasing order."""
    load, out = [0] * ws, [[] for _ in range(ws)]
    for m in sorted(range(len(cells)), key=lambda q: (-cells[q], q)):
        r = min(range(ws), key=lambda q: (load[q], q))
        out[r].append(m)
        load[r] += cells[m]
    return [sorted(x) for x in out]


def ensemble_job(ms, cells, failed, dist=None, device="cpu"):
    """Max-over-ranks ensemble time, total cells of all ranks, and whether
    any rank failed (the same collectives on every rank, failed or not)."""
    import torch
    t = torch.tensor([ms, float(failed)], dtype=torch.float64, device=device)
    c = torch.tensor([float(cells)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), int(c[0]), bool(t[1] > 0)


def ensemble_bench(steps, warmup, ws=1, rank=0, dist=None):
    """64 uneven domains (ip, jp ~ U{96..256}, kp=80, own terrain seed, u* ~
    U[0.2, 0.5]) advanced `steps` steps by one graph launch per step; under
    torchrun the members are sharded over the ranks (shard_members, no
    collective on the data path) and the time is the slowest rank's.  On one
    GPU the same members are also advanced one after another with les_step
    (64 sequential runs).  CUDA events on the launching streams."""
    import torch
    import les_halo_b200 as lh
    E = ENSEMBLE
    doms = ensemble_members()
    mine = shard_members([ip * jp * E["kp"] for ip, jp, _, _ in doms], ws)[rank]
    err, ens_ms, cells, launches, seq_ms, tune = None, float("nan"), 0, 0, None, None
    members, ens = [], None
    try:
        for m in mine:
            ip, jp, ustar, seed = doms[m]
            case = lh.synthetic_case(ip, jp, E["kp"], seed=seed, dt=0.05, nmaxp=50, ustar=ustar)
            g = lh.GpuLes(case)
            g.warmup(1)
            members.append(g)
            cells += ip * jp * E["kp"]
        ens = lh.Ensemble(members)
        ens.step(1, warmup)
        ens.sync()
        st = torch.cuda.ExternalStream(ens.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ens.launches()
        steps = E["steps"]  # the configuration's 200 steps
        e0.record(st)
        ens.step(1 + warmup, steps)
        e1.record(st)
        torch.cuda.synchronize()
        ens_ms = e0.elapsed_time(e1)
        launches = ens.launches() - l0
        tune = ens.tune_info()
        if ws == 1:
            # 64 sequential plain runs: each member in a fresh context with
            # its own autotuned SOR shape and its step graph captured by an
            # untimed step first, one member after another
            seq_ms = 0.0
            for m in mine:
                ip, jp, ustar, seed = doms[m]
                case = lh.synthetic_case(ip, jp, E["kp"], seed=seed, dt=0.05, nmaxp=50, ustar=ustar)
                g = lh.GpuLes(case)
                try:
                    g.warmup(1)
                    g.step(1, 1)
                    g.sync()
                    ms = torch.cuda.ExternalStream(g.stream())
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(ms)
                    g.step(2, E["seq_steps"])
                    b.record(ms)
                    torch.cuda.synchronize()
                    seq_ms += a.elapsed_time(b) * steps / E["seq_steps"]  # per the ensemble's step count
                finally:
                    g.close()
    except Exception as exc:  # reported, never fatal to the headline line
        err = f"{type(exc).__name__}: {exc}"[:300]
    finally:
        if ens is not None:
            ens.close()
        for g in members:
            g.close()
    ens_ms, cells_all, failed = ensemble_job(ens_ms if err is None else float("inf"), cells, err is not None,
                                             dist, "cuda" if dist is not None and dist.get_backend() == "nccl"
                                             else "cpu")
    if failed:
        return {"error": err or "failed on another rank"}
    out = {"members": E["members"], "cells": cells_all, "kp": E["kp"], "steps": steps, "ranks": ws,
           "sharding": "greedy cell-count balance, no collective on the data path",
           "ensemble_mpts": round(cells_all * steps / (ens_ms / 1e3) / 1e6, 1),
           "ensemble_ms_per_step": round(ens_ms / steps, 3), "graph_launches_per_step": 1,
           "kernels_per_step_rank0": int(launches // max(steps, 1)),
           "sor_shape_autotuner": tune,
           "config": f"ip,jp ~ U{{{E['size_lo']}..{E['size_hi']}}}, kp={E['kp']}, u* ~ "
                     f"U[{E['ustar_lo']},{E['ustar_hi']}], seed {E['seed']}"}
    if seq_ms is not None:
        out.update(sequential_mpts=round(cells_all * steps / (seq_ms / 1e3) / 1e6, 1),
                   sequential_ms_per_step=round(seq_ms / steps, 3), speedup=round(seq_ms / ens_ms, 3))
    return out


CONFIG2 = dict(ip=1000, jp=1000, kp=150, seed=1, warm=2, steps=500, chunk=50)


def config2_bench():
    """The mixed-precision pressure configuration: 1000 x 1000 x 150 (1.5e8
    cells; the benchmark terrain generator, 30% plan area), the plain FP32
    step against the FP64-refined press (FP32 SOR sweeps, FP64 rhsav and
    residual sums, FP64 defect corrections with the spectral inner solve to a
    1e-9 relative residual, FP64 pav), both timed with CUDA events on the
    context stream after warm-up steps."""
    import torch
    import les_halo_b200 as lh
    A = CONFIG2
    gpu = None
    try:
        case = lh.synthetic_case(A["ip"], A["jp"], A["kp"], seed=A["seed"], dt=0.05, nmaxp=50)
        cells = A["ip"] * A["jp"] * A["kp"]
        gpu = lh.GpuLes(case)
        del case
        gpu.warmup(1)
        st = torch.cuda.ExternalStream(gpu.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 1
        gpu.step(n, A["warm"])
        n += A["warm"]
        gpu.sync()
        e0.record(st)
        gpu.step(n, A["steps"])
        e1.record(st)
        torch.cuda.synchronize()
        plain_ms = e0.elapsed_time(e1) / A["steps"]
        n += A["steps"]
        gpu.press_refine_fp64(2, 0, 1e-9)
        gpu.step(n, A["warm"])
        n += A["warm"]
        gpu.sync()
        # the configuration's 500 refined steps; the last step of every 50 is
        # checked against the tolerance (its metrics read between chunks)
        worst, most = 0.0, 0
        e0.record(st)
        for c0 in range(0, A["steps"], A["chunk"]):
            gpu.step(n + c0, min(A["chunk"], A["steps"] - c0))
            rmc = gpu.refine_metrics()
            worst, most = max(worst, rmc["rel_final"]), max(most, rmc["outer"])
        e1.record(st)
        torch.cuda.synchronize()
        ref_ms = e0.elapsed_time(e1) / A["steps"]
        rm = gpu.refine_metrics()
        return {"grid": [A["ip"], A["jp"], A["kp"]], "cells": cells, "steps": A["steps"],
                "plain_ms_per_step": round(plain_ms, 3), "plain_mpts": round(cells / plain_ms / 1e3, 1),
                "refined_ms_per_step": round(ref_ms, 3), "refined_mpts": round(cells / ref_ms / 1e3, 1),
                "time_vs_plain": round(ref_ms / plain_ms, 3), "rel_tol": 1e-9,
                "rel_residual_after_fp32_sweeps": rm["rel_initial"], "rel_residual_final": rm["rel_final"],
                "rel_residual_final_worst_sampled": worst, "corrections": rm["outer"],
                "corrections_most_sampled": most, "inner": "spectral (FP64, hand-written mixed-radix FFTs)"}
    except Exception as exc:
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}
    finally:
        if gpu is not None:
            gpu.close()


DECOMP = dict(ranks_one_gpu=2, halo=16, sync_every=8, warm=2, steps=5)


def decomp_bench(ws=1, rank=0, dist=None):
    """The x-decomposed step (les_halo_b200/decomp.py) on the workload: on
    one GPU, DECOMP["ranks_one_gpu"] ranks in this process (device copies
    between their slabs) against the single domain on the same SOR path
    (one-iteration passes; per colour with LES_DD_SOR=colour); under
    torchrun (--decomp), one slab per rank with NCCL
    send/recv and all-reduce, strong scaling of the one domain.  CUDA events
    on the ranks' streams, the slowest rank's time."""
    import torch
    import les_halo_b200 as lh
    from les_halo_b200 import abi, decomp as D
    A = DECOMP
    case = make_case()
    cells, nmaxp, ical = case.ip * case.jp * case.kp, case.params.nmaxp, case.params.ical
    ranks, dd, single_ms = [], None, None
    try:
        if ws == 1:
            dd = D.DecomposedLes(case, A["ranks_one_gpu"], A["halo"], A["sync_every"])
            ranks, ex = dd.ranks, dd.ex
        else:
            slabs = D.split_columns(case.ip, ws, A["halo"])
            r = D.DDRank(case, slabs[rank])
            parts = [None] * ws
            dist.all_gather_object(parts, r.area_part())
            r.set_owned(None if any(x is None for x in parts) else sum(parts))
            ranks, ex = [r], D.DistExchange(r, dist, device="cuda")
        D.run_steps(ranks, ex, 1, A["warm"], nmaxp, ical, A["sync_every"])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s0 = ranks[0].stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        for r in ranks[1:]:
            r.stream().wait_event(e0)
        D.run_steps(ranks, ex, 1 + A["warm"], A["steps"], nmaxp, ical, A["sync_every"])
        for r in ranks[1:]:
            ev = torch.cuda.Event()
            ev.record(r.stream())
            s0.wait_event(ev)
        e1.record(s0)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / A["steps"]
        if dist:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t[0])
        m = ranks[-1].gpu.metrics()
        H, mid = A["halo"], ranks[0]
        per_side = (mid.block_floats(D.STATE_MASK, H) + mid.block_floats(D.RHS_MASK, H) +
                    ((nmaxp - 1) // A["sync_every"]) * mid.block_floats(D.P_MASK, H)) * 4
        for r in ranks:
            r.close()
        ranks = []
        if dd is not None:
            dd.ranks = []
        if ws == 1:
            g = lh.GpuLes(case)
            try:
                if os.environ.get("LES_DD_SOR") == "colour":
                    abi.check(abi.lib().les_ctx_set_sor_path(g.ctx, 1))
                st = torch.cuda.ExternalStream(g.stream())
                g.step(1, A["warm"])
                g.sync()
                e0.record(st)
                g.step(1 + A["warm"], A["steps"])
                e1.record(st)
                torch.cuda.synchronize()
                single_ms = e0.elapsed_time(e1) / A["steps"]
            finally:
                g.close()
        out = {"ranks": A["ranks_one_gpu"] if ws == 1 else ws, "gpus": ws, "halo_columns": H,
               "p_exchange_every": A["sync_every"], "steps": A["steps"], "ms_per_step": round(ms, 3),
               "mpts": round(cells / ms / 1e3, 1), "sor_iters": int(m["sor_iters"]),
               "halo_bytes_per_step_per_neighbour": int(per_side),
               "sor_path": "one-iteration passes, exact all-rank sums"
                           if os.environ.get("LES_DD_SOR") != "colour" else "per colour, exact all-rank sums",
               "transport": "device copies, one process" if ws == 1 else "NCCL send/recv + all-reduce"}
        if single_ms is not None:
            out.update(single_domain_same_path_ms=round(single_ms, 3), time_vs_single=round(ms / single_ms, 3))
        return out
    except Exception as exc:
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}
    finally:
        for r in ranks:
            r.close()


ADJOINT = dict(ip=150, jp=150, kp=90, steps=100, ckpt=10, box=((66, 85), (66, 85), (1, 5)), seed=1)


def adjoint_bench():
    """The adjoint configuration: the 150 x 150 x 90 benchmark terrain from
    its warm-up, 100 steps (all 50 SOR iterations each) with the time-mean
    resolved TKE of a 20 x 20 x 5-cell pedestrian box as the objective, and
    its gradient with respect to the inflow profile, the per-column drag
    scale and the initial state by the device step adjoint with a checkpoint
    every 10 steps (each segment recomputed).  Cost ratio = wall time of the
    gradient (forward with checkpoints, recomputation and adjoint) over the
    forward alone (the same 100 steps with the objective evaluated)."""
    import les_halo_b200 as lh
    A = ADJOINT
    case = lh.synthetic_case(A["ip"], A["jp"], A["kp"], seed=A["seed"], dt=0.05, nmaxp=50)
    case.params.pjuge = -1.0
    gpu = lh.GpuLes(case)
    gpu.warmup(1)
    lh.set_drag(gpu, np.ones((A["ip"], A["jp"]), np.float32))
    nt, ckpt, box = A["steps"], A["ckpt"], A["box"]
    adj = lh.GpuAdjoint(gpu, -(-nt // ckpt) + ckpt + 1, 50)
    try:
        init = adj.nslots - 1
        adj.save(init)
        gpu.step(1, 2)  # capture the step graphs, autotune
        gpu.sync()

        def forward():
            adj.load(init)
            J = 0.0
            for t in range(nt):
                gpu.step(1 + t, 1)
                J += adj.tke(-1, box) / nt
            gpu.sync()
            return J

        forward()
        t0 = time.perf_counter()
        J = forward()
        fwd_s = time.perf_counter() - t0
        adj.load(init)
        lh.tke_gradient(gpu, adj, 1, nt, box, ckpt)  # warm
        adj.load(init)
        gpu.sync()
        t0 = time.perf_counter()
        Jg, g = lh.tke_gradient(gpu, adj, 1, nt, box, ckpt)
        gpu.sync()
        grad_s = time.perf_counter() - t0
        return {"config": f"{A['ip']}x{A['jp']}x{A['kp']}, {nt} steps (SOR 50 each), checkpoint every {ckpt} "
                          "(the last segment's step inputs kept from the forward run, the others recomputed), "
                          f"J = time-mean resolved TKE of box i{box[0]} j{box[1]} k{box[2]}; gradients: inflow "
                          "profile (jp x kp), drag scale (ip x jp), initial state",
                "J": J, "J_in_gradient_run": Jg, "forward_s": round(fwd_s, 4), "gradient_s": round(grad_s, 4),
                "cost_ratio": round(grad_s / fwd_s, 3),
                "adjoint_over_forward": round((grad_s - fwd_s) / fwd_s, 3),
                "grad_wp_norm": float(np.linalg.norm(g["wp"])), "grad_drag_norm": float(np.linalg.norm(g["drag"])),
                "precision": "FP32 fields and adjoint, FP64 objective and parameter-gradient sums"}
    except Exception as exc:
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}
    finally:
        adj.close()
        gpu.close()


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import les_halo_b200 as lh
    from les_halo_b200 import abi

    case = make_case()
    cells = case.ip * case.jp * case.kp
    gpu = lh.GpuLes(case)
    gpu.warmup(1)
    n = 1
    gpu.step(n, args.warmup)
    n += args.warmup
    gpu.sync()
    L = abi.lib()
    # capture the timed step graph (with its event nodes) before timing, then
    # reset the slots so the K timed steps use slots 0..K-1.  Profiling runs
    # (--profile) leave the graph without event nodes.
    if not args.profile:
        abi.check(L.les_ctx_set_timing(gpu.ctx, args.steps))
    gpu.step(n, 1)
    n += 1
    gpu.sync()
    if not args.profile:
        abi.check(L.les_ctx_set_timing(gpu.ctx, args.steps))

    stream = torch.cuda.ExternalStream(gpu.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    launches0 = gpu.launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    ev0.record(stream)
    gpu.step(n, args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    n += args.steps
    if dist:
        dist.barrier()
    ms_total = ev0.elapsed_time(ev1)
    launches = gpu.launches() - launches0
    phases = np.zeros((args.steps, 9), np.float32)
    buf = (C.c_float * 9)()
    for s in range(args.steps if not args.profile else 0):
        abi.check(L.les_ctx_phase_times(gpu.ctx, s, buf, 9))
        phases[s] = np.frombuffer(buf, np.float32)
    m = gpu.metrics()

    # e2e through the C ABI with pinned host buffers: per step the inflow
    # profile goes up, then the step, then the halo round trip of the state
    # arrays (ST_HALO_READ/WRITE of run_LES_kernel) and the step record.
    wp = torch.from_numpy(case.a("wind_profile").ravel(order="F").copy()).pin_memory()
    halos = []
    for h in range(len(abi.HALO_IDS)):
        nf = int(L.les_ctx_halo_floats(gpu.ctx, h))
        halos.append(torch.empty(nf, dtype=torch.float32).pin_memory())
    mrec = abi.LesMetrics()
    e2e_steps = max(3, min(args.steps, 10))
    h2d = wp.numel() * 4 + sum(t.numel() * 4 for t in halos)
    d2h = sum(t.numel() * 4 for t in halos) + C.sizeof(mrec)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        abi.check(L.les_set_wind_profile(gpu.ctx, wp.data_ptr()))
        abi.check(L.les_step(gpu.ctx, n, 1))
        n += 1
        for h, t in enumerate(halos):
            abi.check(L.les_ctx_halo_read(gpu.ctx, h, t.data_ptr()))
        for h, t in enumerate(halos):
            abi.check(L.les_ctx_halo_write(gpu.ctx, h, t.data_ptr()))
        abi.check(L.les_last_metrics(gpu.ctx, C.byref(mrec)))
    e2e_s = time.perf_counter() - t0

    # aveflow.f95:72-88 on the device-resident state (main_ocl.f95:313 calls
    # it after every step), timed alone with CUDA events: one call starts
    # the sums (allocating them), then K accumulating calls.  The ten sums
    # (1.7 GB at 600x600x120) are far larger than L2.
    ave_k = max(3, min(args.steps, 10))
    big = 1 << 30
    gpu.aveflow(1, 1, big)
    torch.cuda.synchronize()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for s in range(ave_k):
        gpu.aveflow(2 + s, 1, big)
    ev3.record(stream)
    torch.cuda.synchronize()
    ave_ms = ev2.elapsed_time(ev3) / ave_k

    # FP64-refined press on the same state: the plain FP32 sweeps, then up to
    # REFINE["outer"] FP64 defect corrections (spectral inner solve) until the
    # FP64 relative residual is at most REFINE["tol"], FP64 pav; CUDA events
    # around ref_k steps.
    refined = None
    if not args.profile and args.refine:
        try:
            outer, inner, tol = REFINE["outer"], REFINE["inner"], REFINE["tol"]
            abi.check(L.les_press_refine_fp64(gpu.ctx, outer, inner, tol))
            gpu.step(n, 1)
            n += 1
            ref_k = max(3, min(args.steps, 5))
            torch.cuda.synchronize()
            ev2.record(stream)
            gpu.step(n, ref_k)
            ev3.record(stream)
            torch.cuda.synchronize()
            n += ref_k
            ref_ms = ev2.elapsed_time(ev3) / ref_k
            rm = gpu.refine_metrics()
            abi.check(L.les_press_refine_fp64(gpu.ctx, 0, 0, 0.0))
            refined = {"outer": outer, "inner": "spectral (FP64)" if inner == 0 else f"{inner} SOR iterations",
                       "rel_tol": tol, "ms_per_step": round(ref_ms, 4),
                       "mpts": round(cells / (ref_ms / 1e3) / 1e6, 1), "steps": ref_k,
                       "rel_residual_after_fp32_sweeps": rm["rel_initial"],
                       "rel_residual_final": rm["rel_final"], "corrections": rm["outer"]}
        except Exception as exc:
            refined = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    ms_total, e2e_s, value, e2e_val = job_rates(ms_total, e2e_s, cells, args.steps, e2e_steps, ws,
                                                dist, "cuda")
    ms_step = ms_total / args.steps

    sor_launch_ms = float(np.mean(phases[:, 5])) if not args.profile else float("nan")
    peak, peak_kind = _peaks()
    ipl = float(L.les_ctx_sor_iters_per_launch(gpu.ctx))
    sh = [C.c_int() for _ in range(4)]
    abi.check(L.les_ctx_sor_shape(gpu.ctx, *[C.byref(x) for x in sh]))
    tT, tY, tX, tK = (x.value for x in sh)
    rw = C.c_int()
    abi.check(L.les_ctx_sor_rows(gpu.ctx, C.byref(rw)))
    achieved = SOR_BYTES_PER_CELL_PER_ITER * ipl * cells / (sor_launch_ms / 1e3) / 1e9
    step_gbs = STEP_BYTES_PER_CELL * cells / (ms_step / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "sor_traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get("bytes_per_launch")
        except Exception:
            traffic = None
    # every rank takes part (its shard of the members, and the collectives)
    ens_line = None
    if not args.profile and not args.no_ensemble:
        ens_line = ensemble_bench(args.steps, args.warmup, ws, rank, dist)
    dd_line = decomp_bench(ws, rank, dist) if (ws > 1 and args.decomp and not args.profile) else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mpts/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded terrain + log-law inflow)",
            "config": {"workload": workload_desc(case.ip, case.jp, case.kp),
                       "grid": [case.ip, case.jp, case.kp], "sor_iters": int(m["sor_iters"]),
                       "parallelism": f"replicas x{ws}",
                       "sor_tile": {"iters_per_pass": tT, "rows": tY, "cols": tX, "k_chunks": tK,
                                    "rows_per_warp": rw.value},
                       "l2": "inputs larger than L2 (19 state fields, 3.5 GB)"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm",
                         "kernel": ("k_sor_colour" if ipl < 1 else "k_sor1p" if rw.value == 2 else
                                    {1: "k_sor1", 2: "k_sor2"}.get(tT, "k_sor_tb")),
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic": f"{SOR_BYTES_PER_CELL_PER_ITER} B/cell/iteration x {ipl} iterations "
                                        f"per launch x {cells} cells"},
            "step_roofline": {"achieved_gbs": round(step_gbs, 1), "frac": round(step_gbs / peak, 4),
                              "bytes_per_cell": STEP_BYTES_PER_CELL},
            "phases_ms": {k: round(float(v), 4) for k, v in zip(
                ["velnw_bondv1", "velfg_feedbf_sm", "boundsm_visc_adam", "rhs_rhsav", "gap",
                 "sor_first_launch", "sor_rest", "pav", "step"], phases.mean(axis=0))},
            "e2e": {"value": round(e2e_val, 3), "unit": "Mpts/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "path": "C ABI: les_set_wind_profile + les_step + les_ctx_halo_read/write x7 + "
                            "les_last_metrics, pinned host buffers, wall clock"},
            "clocks": clocks,
            "refined_press": dict(refined, time_vs_plain=round(refined["ms_per_step"] / ms_step, 3))
            if refined and "ms_per_step" in refined else refined,
            "aveflow": {"kernel": "k_ave_accum4" if case.ip % 4 == 0 else "k_ave_accum",
                        "ms_per_call": round(ave_ms, 4),
                        "achieved": round(AVE_BYTES_PER_CELL * cells / (ave_ms / 1e3) / 1e9, 1),
                        "peak": peak, "unit": "GB/s",
                        "frac": round(AVE_BYTES_PER_CELL * cells / (ave_ms / 1e3) / 1e9 / peak, 4),
                        "bytes_per_cell": AVE_BYTES_PER_CELL, "calls": ave_k},
        }
        if ens_line is not None:
            line["ensemble"] = ens_line
        if dd_line is not None:
            line["decomposition"] = dd_line
        if not args.profile and not args.no_adjoint and ws == 1:
            line["adjoint"] = adjoint_bench()
        if not args.profile and args.refine and not args.no_config2 and ws == 1:
            line["config2_refined_press"] = config2_bench()
        if not args.profile and not args.no_decomp and ws == 1:
            line["decomposition"] = decomp_bench()
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(os.cpu_count() or 1)
        print(json.dumps(line), flush=True)
    gpu.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-refine", dest="refine", action="store_false",
                    help="skip the FP64-refined press measurement")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 64-domain ensemble measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint (config-3) cost measurement")
    ap.add_argument("--no-config2", action="store_true",
                    help="skip the 1000x1000x150 refined-press measurement")
    ap.add_argument("--no-decomp", action="store_true",
                    help="skip the x-decomposed step measurement (one GPU: ranks in one process)")
    ap.add_argument("--decomp", action="store_true",
                    help="under torchrun: also time the one domain decomposed over the ranks (NCCL)")
    ap.add_argument("--profile", action="store_true",
                    help="no in-graph timing events (for runs under ncu)")
    ap.add_argument("--grid", default=None,
                    help="IP,JP,KP: run a smaller grid (profiling captures); the line names it")
    args = ap.parse_args()
    if args.grid:
        ip, jp, kp = (int(x) for x in args.grid.split(","))
        WORKLOAD.update(ip=ip, jp=jp, kp=kp)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
