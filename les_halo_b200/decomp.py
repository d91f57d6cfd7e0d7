"""x-decomposed LES domain: one context per rank over a slab of columns.

The reference runs its domain on one device and only round-trips its halos
through the ST_HALO_READ_* / ST_HALO_WRITE_* states
(src/OpenCL/module_LES_combined_ocl_TEMPL_V2.f95:438-491) in the ring format
of src/OpenCL/Kernels/halo_exchange.cl:3-291.  Here the domain splits into
slabs along x (i): rank r owns a run of columns and holds up to ``halo``
columns of each neighbour beside them, which it recomputes along with its
own and refreshes from the owner by exchanges of the W/E halo blocks (the
phase schedule is in include/les_abi.h beside les_dd_phase).  The global
sums travel as the limbs of their exact Q63.64 totals, so every own cell
stays the single domain's bit for bit.

Transports: ``LocalExchange`` (every rank in this process on one GPU, halo
blocks ordered by CUDA events between the ranks' streams, the sums added by
one kernel) and ``DistExchange`` (one rank per process, NCCL send/recv and
all-reduce through torch.distributed; with gloo and CPU tensors the same
code exercises the host logic).
"""
from __future__ import annotations

import contextlib
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from . import fields as FL
from .model import GpuLes, LesCase, _copy_params

STATE_FIELDS = ["u", "v", "w", "p", "f", "g", "h", "usum", "vsum", "wsum", "fold", "gold", "hold"]
DEFAULT_HALO = 16
DEFAULT_SYNC = 8
NLIMBS = 6


def field_mask(names) -> int:
    m = 0
    for n in names:
        m |= 1 << abi.FIELD_IDS.index(n)
    return m


STATE_MASK = field_mask(STATE_FIELDS)
RHS_MASK = field_mask(["rhs"])
P_MASK = field_mask(["p"])


@dataclass
class Slab:
    """Rank `rank`'s columns: local column l is global column l + off; the
    context has `im` columns, of which olo..ohi (local) are its own."""
    rank: int
    nranks: int
    off: int
    im: int
    olo: int
    ohi: int
    halo: int

    @property
    def west(self):
        return self.rank - 1 if self.rank > 0 else None

    @property
    def east(self):
        return self.rank + 1 if self.rank < self.nranks - 1 else None

    @property
    def own_global(self):
        return self.olo + self.off, self.ohi + self.off


def split_columns(ip: int, nranks: int, halo: int = DEFAULT_HALO):
    """Slabs of an ip-column domain over nranks ranks.  Own widths are even
    (but the last) and the halo even, so every slab starts on an even global
    offset and the SOR colour of a local cell, (i+j+k+nrd) odd
    (press.f95:155), is the global cell's."""
    if nranks < 1 or halo < 0 or halo % 2:
        raise ValueError("need nranks >= 1 and an even halo width")
    base = (ip // nranks) // 2 * 2
    widths = [base] * (nranks - 1) + [ip - base * (nranks - 1)]
    if nranks > 1 and min(widths) < max(halo, 2):
        raise ValueError(f"{ip} columns over {nranks} ranks leave fewer own columns than the halo ({halo})")
    slabs, a = [], 1
    for r, w in enumerate(widths):
        b = a + w - 1
        lo = a - (halo if r > 0 else 0)
        hi = b + (halo if r < nranks - 1 else 0)
        off = lo - 1
        slabs.append(Slab(r, nranks, off, hi - lo + 1, a - off, b - off, halo))
        a = b + 1
    return slabs


def slab_case(case: LesCase, slab: Slab) -> LesCase:
    """The slab's arrays (every array with an i dimension cut to the slab's
    columns and ghosts; the rest copied) and parameters (ip = slab width)."""
    ip, jp, kp = case.ip, case.jp, case.kp
    prm = _copy_params(case.params)
    prm.ip = slab.im
    out = LesCase(slab.im, jp, kp, prm, {}, case.built_fraction)
    for name, arr in case.arrays.items():
        if "ip" not in FL._BOUNDS[name][0]:
            out.arrays[name] = arr.copy(order="F")
            continue
        (glo, ghi) = FL.bounds(name, ip, jp, kp)[0]
        (llo, lhi) = FL.bounds(name, slab.im, jp, kp)[0]
        a, b = llo + slab.off - glo, lhi + slab.off - glo + 1
        if a < 0 or b > ghi - glo + 1:
            raise ValueError(f"slab columns of {name} fall outside the domain")
        out.arrays[name] = np.asfortranarray(arr[a:b])
    return out


class DDRank:
    """One rank's context (a GpuLes over its slab, les_dd_set_owned applied
    with the whole domain's rhsav/pav denominator)."""

    def __init__(self, case: LesCase, slab: Slab):
        self.slab = slab
        self.gpu = GpuLes(slab_case(case, slab))
        self.ctx = self.gpu.ctx
        self._sums = None
        self._stream = None

    def area_part(self) -> int:
        lo, hi, bad = C.c_ulonglong(), C.c_longlong(), C.c_int()
        abi.check(abi.lib().les_dd_area_part(self.ctx, self.slab.olo, self.slab.ohi, C.byref(lo), C.byref(hi),
                                             C.byref(bad)))
        return None if bad.value else (hi.value << 64) + lo.value

    def set_owned(self, area_total):
        bad = area_total is None
        t = 0 if bad else area_total
        abi.check(abi.lib().les_dd_set_owned(self.ctx, self.slab.olo, self.slab.ohi, t & (2**64 - 1),
                                             t >> 64, int(bad)))

    # -- what the transports use --
    def stream(self):
        if self._stream is None:
            import torch
            self._stream = torch.cuda.ExternalStream(self.gpu.stream())
        return self._stream

    def sums(self):
        """The context's limbs (int64[6] on the device) as a torch tensor."""
        if self._sums is None:
            import torch
            d = C.c_void_p()
            abi.check(abi.lib().les_dd_sums(self.ctx, C.byref(d)))
            self._sums = torch.as_tensor(_DevArray(d.value, NLIMBS, "<i8"), device="cuda")
        return self._sums

    def block_floats(self, mask, width) -> int:
        return int(abi.lib().les_dd_block_floats(self.ctx, mask, width))

    def pack(self, mask, i0, width, buf):
        abi.check(abi.lib().les_dd_pack(self.ctx, mask, i0, width, C.c_void_p(buf.data_ptr())))

    def unpack(self, mask, i0, width, buf):
        abi.check(abi.lib().les_dd_unpack(self.ctx, mask, i0, width, C.c_void_p(buf.data_ptr())))

    def phase(self, ph, arg=0):
        abi.check(abi.lib().les_dd_phase(self.ctx, ph, arg))

    def close(self):
        self._sums = None
        self.gpu.close()


class _DevArray:
    """A device buffer described by __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


def _transfers(slabs, halo):
    """(src rank, dst rank, src first column, dst first column) of every
    halo block: each rank's H own columns next to a neighbour go into that
    neighbour's halo."""
    out = []
    for s in slabs:
        if s.east is not None:
            e = slabs[s.east]
            out.append((s.rank, e.rank, s.ohi - halo + 1, e.olo - halo))  # eastward
            out.append((e.rank, s.rank, e.olo, s.ohi + 1))                 # westward
    return out


class LocalExchange:
    """Every rank in this process: a halo block is packed on the owner's
    stream, unpacked on the neighbour's after a CUDA event, and the sums are
    added by one kernel on rank 0's stream (les_dd_local_sum)."""

    def __init__(self, ranks):
        import torch
        self.torch = torch
        self.ranks = ranks
        self.halo = ranks[0].slab.halo
        self.xfers = _transfers([r.slab for r in ranks], self.halo)
        self.bufs = {}
        self._ctxs = (C.c_void_p * len(ranks))(*[r.ctx.value for r in ranks])

    def _buf(self, key, n, device):
        b = self.bufs.get(key)
        if b is None or b[0].numel() < n:
            b = [self.torch.empty(n, dtype=self.torch.float32, device=device), None]
            self.bufs[key] = b
        return b

    def exchange(self, mask):
        torch = self.torch
        if self.halo == 0:
            return
        for q, (s, d, si0, di0) in enumerate(self.xfers):
            src, dst = self.ranks[s], self.ranks[d]
            n = src.block_floats(mask, self.halo)
            b = self._buf((q, mask), n, torch.device("cuda", torch.cuda.current_device()))
            if b[1] is not None:
                src.stream().wait_event(b[1])  # the last unpack from this buffer is done
            src.pack(mask, si0, self.halo, b[0])
            ev = torch.cuda.Event()
            ev.record(src.stream())
            dst.stream().wait_event(ev)
            dst.unpack(mask, di0, self.halo, b[0])
            b[1] = torch.cuda.Event()
            b[1].record(dst.stream())

    def allreduce(self):
        if len(self.ranks) > 1:
            abi.check(abi.lib().les_dd_local_sum(len(self.ranks), self._ctxs))


class DistExchange:
    """One rank per process over torch.distributed (NCCL for the product,
    gloo with CPU tensors in the host tests).  Each exchange is one batch of
    send/recv pairs with the two neighbours; the sums are one all-reduce.
    device="cpu" with a GPU rank stages the blocks and the sums through host
    memory (gloo between processes that share a GPU)."""

    def __init__(self, rank, dist, device=None):
        import torch
        self.torch = torch
        self.rank = rank
        self.dist = dist
        self.halo = rank.slab.halo
        self.device = device
        self.stage = device == "cpu" and rank.stream() is not None
        self.bufs = {}

    def _ctx(self):
        s = self.rank.stream()
        return self.torch.cuda.stream(s) if s is not None else contextlib.nullcontext()

    def _buf(self, key, n, device=None):
        b = self.bufs.get(key)
        if b is None or b.numel() < n:
            b = self.torch.empty(n, dtype=self.torch.float32, device=device or self.device)
            self.bufs[key] = b
        return b

    def exchange(self, mask):
        s, dist, H = self.rank.slab, self.dist, self.halo
        if H == 0 or s.nranks == 1:
            return
        n = self.rank.block_floats(mask, H)
        with self._ctx():
            ops, recvs = [], []
            for side, nb, si0, di0 in (("e", s.east, s.ohi - H + 1, s.ohi + 1), ("w", s.west, s.olo, s.olo - H)):
                if nb is None:
                    continue
                sb, rb = self._buf(("s", side, mask), n), self._buf(("r", side, mask), n)
                if self.stage:
                    db = self._buf(("d", side, mask), n, "cuda")
                    self.rank.pack(mask, si0, H, db)
                    sb[:n].copy_(db[:n])  # device to host, ordered after the pack
                else:
                    self.rank.pack(mask, si0, H, sb)
                ops += [dist.P2POp(dist.isend, sb[:n], nb), dist.P2POp(dist.irecv, rb[:n], nb)]
                recvs.append((side, di0, rb))
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            for side, di0, rb in recvs:
                if self.stage:
                    db = self._buf(("d", side, mask), n, "cuda")
                    db[:n].copy_(rb[:n])
                    rb = db
                self.rank.unpack(mask, di0, H, rb)

    def allreduce(self):
        with self._ctx():
            if self.stage:
                t = self.rank.sums().cpu()
                self.dist.all_reduce(t)
                self.rank.sums().copy_(t)
            else:
                self.dist.all_reduce(self.rank.sums())


def run_steps(ranks, ex, n0: int, nsteps: int, nmaxp: int, ical: int = 0, sync_every: int = DEFAULT_SYNC):
    """Steps n0 .. n0+nsteps-1 of the ranks in this process (all of them for
    LocalExchange, this process's one for DistExchange), the schedule of
    les_dd_phase (include/les_abi.h)."""
    if sync_every < 1:
        raise ValueError("sync_every >= 1")
    for s in range(nsteps):
        n = n0 + s
        for r in ranks:
            r.phase(abi.LES_DD_BEGIN, n)
        ex.exchange(STATE_MASK)
        for r in ranks:
            r.phase(abi.LES_DD_MOMENTUM, 1 if (n == 1 and ical == 0) else 2)
        ex.allreduce()
        for r in ranks:
            r.phase(abi.LES_DD_RHSAV)
        ex.exchange(RHS_MASK)
        for it in range(nmaxp):
            if it and it % sync_every == 0:
                ex.exchange(P_MASK)
            for r in ranks:
                r.phase(abi.LES_DD_SOR_ITER)
            ex.allreduce()
            for r in ranks:
                r.phase(abi.LES_DD_SOR_TEST)
        for r in ranks:
            r.phase(abi.LES_DD_PAV_SUM)
        ex.allreduce()
        for r in ranks:
            r.phase(abi.LES_DD_PAV_END)


class DecomposedLes:
    """Every rank of an x-decomposed domain in this process (LocalExchange):
    the single-GPU (or one-process) driver and the test harness."""

    def __init__(self, case: LesCase, nranks: int, halo: int = DEFAULT_HALO, sync_every: int = DEFAULT_SYNC):
        if 2 * sync_every > halo and nranks > 1:
            raise ValueError("sync_every <= halo / 2: an SOR iteration moves the slab-edge error 2 columns")
        self.case = case
        self.slabs = split_columns(case.ip, nranks, halo if nranks > 1 else 0)
        self.sync_every = sync_every
        self.ranks = [DDRank(case, s) for s in self.slabs]
        parts = [r.area_part() for r in self.ranks]
        total = None if any(p is None for p in parts) else sum(parts)
        for r in self.ranks:
            r.set_owned(total)
        self.ex = LocalExchange(self.ranks)

    def step(self, n0, nsteps=1):
        run_steps(self.ranks, self.ex, n0, nsteps, self.case.params.nmaxp, self.case.params.ical, self.sync_every)

    def sync(self):
        for r in self.ranks:
            r.gpu.sync()

    def download(self, names):
        """Global Fortran-layout arrays assembled from every rank's own
        columns (ghost columns of the domain from the end ranks)."""
        ip, jp, kp = self.case.ip, self.case.jp, self.case.kp
        out = {n: FL.alloc(n, ip, jp, kp) for n in names}
        for r in self.ranks:
            loc = r.gpu.download(names)
            s = r.slab
            for n in names:
                (glo, ghi) = FL.bounds(n, ip, jp, kp)[0]
                (llo, lhi) = FL.bounds(n, s.im, jp, kp)[0]
                a = s.olo if s.west is not None else llo   # local column range this rank supplies
                b = s.ohi if s.east is not None else lhi
                out[n][a + s.off - glo:b + s.off - glo + 1] = loc[n][a - llo:b - llo + 1]
        return out

    def metrics(self):
        return [r.gpu.metrics() for r in self.ranks]

    def close(self):
        for r in self.ranks:
            r.close()
        self.ranks = []
