"""Host logic of the x-decomposed domain (les_halo_b200/decomp.py) on CPU:
the column split, the slab arrays, and the exchange and phase schedule over
three gloo ranks whose "contexts" are numpy boxes (no GPU; the device path
is tests/test_gpu_decomp.py)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from les_halo_b200 import abi, decomp as D, fields as FL


@pytest.mark.parametrize("ip,n,h", [(100, 3, 16), (64, 2, 12), (37, 1, 0), (300, 8, 16), (98, 4, 2)])
def test_split_columns_covers_the_domain(ip, n, h):
    slabs = D.split_columns(ip, n, h)
    own = []
    for s in slabs:
        a, b = s.own_global
        own += list(range(a, b + 1))
        assert s.off % 2 == 0                      # SOR colours agree with the global cells
        assert 1 <= s.olo <= s.ohi <= s.im
        assert s.olo == (1 if s.west is None else h + 1)
        assert s.im - s.ohi == (0 if s.east is None else h)
        assert s.ohi - s.olo + 1 >= h
    assert own == list(range(1, ip + 1))


def test_split_rejects_narrow_slabs_and_odd_halos():
    with pytest.raises(ValueError):
        D.split_columns(40, 4, 16)
    with pytest.raises(ValueError):
        D.split_columns(100, 2, 5)


def test_slab_arrays_are_the_domain_columns():
    from les_halo_b200 import synthetic_case
    case = synthetic_case(60, 12, 10, seed=4, masks_and_poisson=lambda c, zbm: None)
    rng = np.random.default_rng(1)
    for n in FL.STATE + FL.MASKS + ["cn1", "cn2l", "cn2s"]:
        case.arrays[n][...] = rng.standard_normal(case.arrays[n].shape).astype(np.float32)
    for s in D.split_columns(60, 3, 8):
        sc = D.slab_case(case, s)
        assert (sc.ip, sc.params.ip, sc.jp, sc.kp) == (s.im, s.im, 12, 10)
        for n, a in sc.arrays.items():
            g = case.arrays[n]
            if "ip" not in FL._BOUNDS[n][0]:
                assert np.array_equal(a, g)
                continue
            (glo, _), (llo, lhi) = FL.bounds(n, 60, 12, 10)[0], FL.bounds(n, s.im, 12, 10)[0]
            assert a.shape == (lhi - llo + 1,) + g.shape[1:]
            for i in (llo, s.olo, s.ohi, lhi):   # local column i is global column i + off
                assert np.array_equal(a[i - llo], g[i + s.off - glo]), (n, i)


class FakeRank:
    """A rank whose fields are numpy boxes [column + 2, row] (4 rows): own
    columns hold 100 * global column + field id, halo columns -1."""
    ROWS = 4

    def __init__(self, slab, log):
        import torch
        self.torch = torch
        self.slab, self.log = slab, log
        self.box = {}
        for f in range(len(abi.FIELD_IDS)):
            b = np.full((slab.im + 4, self.ROWS), -1.0, dtype=np.float32)
            for i in range(slab.olo, slab.ohi + 1):
                b[i + 2] = 100.0 * (i + slab.off) + f
            self.box[f] = b
        self._sums = torch.tensor([slab.rank + 1, 2 * slab.rank, 7, -1, 0, 0], dtype=torch.int64)

    def stream(self):
        return None

    def sums(self):
        return self._sums

    def block_floats(self, mask, width):
        return bin(mask).count("1") * width * self.ROWS

    def _fields(self, mask):
        return [f for f in range(len(abi.FIELD_IDS)) if mask >> f & 1]

    def pack(self, mask, i0, width, buf):
        vals = [self.box[f][i0 + 2:i0 + 2 + width].T for f in self._fields(mask)]  # row-major, column fastest
        buf[:self.block_floats(mask, width)] = self.torch.from_numpy(np.concatenate([v.ravel() for v in vals]))
        self.log.append(("pack", mask, i0))

    def unpack(self, mask, i0, width, buf):
        v = buf[:self.block_floats(mask, width)].numpy().reshape(-1, self.ROWS, width)
        for q, f in enumerate(self._fields(mask)):
            self.box[f][i0 + 2:i0 + 2 + width] = v[q].T
        self.log.append(("unpack", mask, i0))

    def phase(self, ph, arg=0):
        self.log.append(("phase", ph, arg))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, nranks, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=nranks, timeout=datetime.timedelta(seconds=60))
    try:
        slab = D.split_columns(40, nranks, 6)[rank]
        log = []
        fr = FakeRank(slab, log)
        ex = D.DistExchange(fr, dist, device="cpu")
        # one exchange of a field subset: halo columns take the owner's values
        ex.exchange(D.field_mask(["u", "p", "hold"]))
        lo, hi = slab.olo - (6 if slab.west is not None else 0), slab.ohi + (6 if slab.east is not None else 0)
        got = {f: fr.box[f][lo + 2:hi + 3, 0].tolist() for f in range(len(abi.FIELD_IDS))}
        ex.allreduce()
        sums = fr.sums().tolist()
        del log[:]
        D.run_steps([fr], ex, 1, 2, nmaxp=5, ical=0, sync_every=2)
        q.put((rank, slab, lo, hi, got, sums, list(log)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_exchange_halos_and_sum_limbs():
    n = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, n, port, q)) for r in range(n)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = {r[0]: r[1:] for r in (q.get(timeout=10) for _ in range(n))}
    mask_fields = {abi.FIELD_IDS.index(x) for x in ("u", "p", "hold")}
    for r, (slab, lo, hi, got, sums, log) in res.items():
        for f, col in got.items():
            for q_, i in enumerate(range(lo, hi + 1)):
                own = slab.olo <= i <= slab.ohi
                want = 100.0 * (i + slab.off) + f if (own or f in mask_fields) else -1.0
                assert col[q_] == want, (r, f, i)
        assert sums == [1 + 2 + 3, 0 + 2 + 4, 21, -3, 0, 0]
        # the phase schedule of one step: begin, state halo, momentum, sum,
        # rhsav, rhs halo, 5 SOR iterations (p halo before the 3rd and 5th), pav
        P = abi
        step = lambda n: ([("phase", P.LES_DD_BEGIN, n)] + _x(slab, D.STATE_MASK) +
                          [("phase", P.LES_DD_MOMENTUM, 1 if n == 1 else 2), ("phase", P.LES_DD_RHSAV, 0)] +
                          _x(slab, D.RHS_MASK) +
                          sum([(_x(slab, D.P_MASK) if it in (2, 4) else []) +
                               [("phase", P.LES_DD_SOR_ITER, 0), ("phase", P.LES_DD_SOR_TEST, 0)]
                               for it in range(5)], []) +
                          [("phase", P.LES_DD_PAV_SUM, 0), ("phase", P.LES_DD_PAV_END, 0)])
        assert log == step(1) + step(2), r


def _x(slab, mask):
    """Pack / unpack calls of one exchange on this rank: east side first."""
    out = []
    if slab.east is not None:
        out.append(("pack", mask, slab.ohi - slab.halo + 1))
    if slab.west is not None:
        out.append(("pack", mask, slab.olo))
    if slab.east is not None:
        out.append(("unpack", mask, slab.ohi + 1))
    if slab.west is not None:
        out.append(("unpack", mask, slab.olo - slab.halo))
    return out


def test_dd_entries_validate_without_a_gpu():
    import ctypes as C
    L = abi.lib()
    lo, hi, bad = C.c_ulonglong(), C.c_longlong(), C.c_int()
    assert L.les_dd_area_part(None, 1, 2, C.byref(lo), C.byref(hi), C.byref(bad)) == abi.LES_ERR_BAD_ARG
    assert L.les_dd_set_owned(None, 1, 2, 0, 0, 0) == abi.LES_ERR_BAD_ARG
    assert L.les_dd_phase(None, abi.LES_DD_BEGIN, 1) == abi.LES_ERR_BAD_ARG
    assert L.les_dd_pack(None, D.P_MASK, 1, 4, None) == abi.LES_ERR_BAD_ARG
    assert L.les_dd_unpack(None, D.P_MASK, 1, 4, None) == abi.LES_ERR_BAD_ARG
    assert L.les_dd_block_floats(None, D.P_MASK, 4) == -1
    d = C.c_void_p()
    assert L.les_dd_sums(None, C.byref(d)) == abi.LES_ERR_BAD_ARG
