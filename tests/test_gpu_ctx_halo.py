"""The context's halo entries (les_ctx_halo_read / les_ctx_halo_write) on
the reference's combined arrays, bit for bit against the oracle.

run_LES_kernel exchanges the state through the halo rings of the combined
arrays p2, uvw, uvwsum, fgh, fgh_old, rhs and sm
(src/OpenCL/module_LES_combined_ocl_TEMPL_V2.f95:111-143).  The expected
buffers are the oracle's halo_exchange.cl restatement applied to combined
arrays built from the downloaded fields the way module_LES_conversions.f95
builds them (convert_to_uvw :3-24 with its k = -1 rule at :18-21,
convert_to_fgh :26-38, convert_to_fgh_old :40-53); p2 is (p, p).
"""
import numpy as np
import pytest

import oracle
from les_halo_b200 import GpuLes, abi, fields as FL, synthetic_case

pytestmark = pytest.mark.gpu
NAMES = FL.STATE


def _combined(which, F, ip, jp, kp):
    """(vdim, extents, AoS array in Fortran order, v fastest) of one combined array."""
    def stack(comps, shape):
        out = np.zeros((len(comps),) + shape, np.float32, order="F")
        for v, c in enumerate(comps):
            if c is not None:
                out[v] = c
        return out
    if which == "p":
        return 2, (ip + 3, jp + 3, kp + 2), stack([F["p"], F["p"]], (ip + 3, jp + 3, kp + 2))
    if which == "uvw":
        shape = (ip + 2, jp + 3, kp + 3)  # (0:ip+1, -1:jp+1, -1:kp+1)
        a = np.zeros((4,) + shape, np.float32, order="F")
        a[0, :, :, 1:] = F["u"]  # u, v: 0:kp+1; their k = -1 entries stay 0 (:18-21)
        a[1, :, :, 1:] = F["v"]
        a[2] = F["w"]
        return 4, shape, a
    if which in ("uvwsum", "fgh"):
        names = ("usum", "vsum", "wsum") if which == "uvwsum" else ("f", "g", "h")
        shape = (ip + 1, jp + 1, kp + 1)
        return 4, shape, stack([F[n] for n in names] + [None], shape)
    if which == "fgh_old":
        shape = (ip, jp, kp)
        return 4, shape, stack([F["fold"], F["gold"], F["hold"], None], shape)
    if which == "rhs":
        return 1, (ip + 2, jp + 2, kp + 2), F["rhs"][None]
    if which == "sm":
        return 1, (ip + 3, jp + 3, kp + 2), F["sm"][None]
    raise KeyError(which)


def _fields_from(which, comb, F):
    """Write a combined array's components back into field copies (convert_from_*)."""
    F = {k: v.copy(order="F") for k, v in F.items()}
    if which == "p":
        F["p"] = comb[0].copy(order="F")
    elif which == "uvw":
        F["u"], F["v"], F["w"] = (comb[0, :, :, 1:].copy(order="F"), comb[1, :, :, 1:].copy(order="F"),
                                  comb[2].copy(order="F"))
    elif which in ("uvwsum", "fgh", "fgh_old"):
        names = {"uvwsum": ("usum", "vsum", "wsum"), "fgh": ("f", "g", "h"),
                 "fgh_old": ("fold", "gold", "hold")}[which]
        for v, n in enumerate(names):
            F[n] = comb[v].copy(order="F")
    else:
        F[which] = comb[0].copy(order="F")
    return F


# run_LES_kernel's halo buffer sizes, TEMPL:113-119 with h_w = 1
def _ref_sizes(ip, jp, kp):
    return {"p": 4 * (ip + jp + 4) * (kp + 2), "uvw": 8 * (ip + jp + 3) * (kp + 3),
            "uvwsum": 8 * (ip + jp) * (kp + 1), "fgh": 8 * (ip + jp) * (kp + 1),
            "fgh_old": 8 * (ip + jp - 2) * kp, "rhs": 2 * (ip + jp + 2) * (kp + 2),
            "sm": 2 * (ip + jp + 4) * (kp + 2)}


_KEEP = []


def _host(n, pinned, fill=0.0):
    """A float32 host buffer: pageable numpy memory (staged through the
    device by the library), or page-locked memory (torch pin_memory), which
    the library's kernel reads and writes in place."""
    if not pinned:
        return np.full(n, fill, np.float32)
    import torch
    t = torch.full((n,), fill, dtype=torch.float32).pin_memory()
    _KEEP.append(t)
    return t.numpy()


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("dims", [(24, 20, 16), (33, 19, 12)])
def test_ctx_halo_read_write_vs_oracle(require_gpu, dims, pinned):
    ip, jp, kp = dims
    L = abi.lib()
    case = synthetic_case(ip, jp, kp, seed=ip + jp, masks_and_poisson=oracle.masks_and_poisson)
    gpu = GpuLes(case)
    gpu.warmup(1)
    gpu.step(1, 2)
    F = gpu.download(NAMES)
    rng = np.random.default_rng(ip)
    sizes = _ref_sizes(ip, jp, kp)
    for h, which in enumerate(abi.HALO_IDS):
        vd, (im, jm, km), comb = _combined(which, F, ip, jp, kp)
        n = int(L.les_ctx_halo_floats(gpu.ctx, h))
        assert n == oracle.halo_buffer_floats(im, jm, km, 1, vd) == sizes[which], which
        # read: the ring of the combined array, N|S|W|E, component-major
        want = np.zeros(n, np.float32)
        oracle.halo_pack(np.ascontiguousarray(comb.ravel(order="F")), want, im, jm, km, 1, vd)
        got = _host(n, pinned, np.nan)
        abi.check(L.les_ctx_halo_read(gpu.ctx, h, got.ctypes.data))
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=which)
        # write: random ring values land where halo_exchange.cl's write puts them
        buf = _host(n, pinned)
        buf[:] = rng.standard_normal(n).astype(np.float32)
        flat = np.ascontiguousarray(comb.ravel(order="F"))
        oracle.halo_unpack(flat, np.ascontiguousarray(buf), im, jm, km, 1, vd)
        after = flat.reshape(comb.shape, order="F")
        expect = _fields_from(which, after, F)
        abi.check(L.les_ctx_halo_write(gpu.ctx, h, buf.ctypes.data))
        now = gpu.download(NAMES)
        for nm in NAMES:
            np.testing.assert_array_equal(now[nm].view(np.uint32), expect[nm].view(np.uint32),
                                          err_msg=f"{which}: {nm}")
        # round trip: reading the ring back gives what a read of the new
        # state must give, and writing it again changes nothing
        back = _host(n, pinned)
        abi.check(L.les_ctx_halo_read(gpu.ctx, h, back.ctypes.data))
        _, _, comb2 = _combined(which, now, ip, jp, kp)
        want2 = np.zeros(n, np.float32)
        oracle.halo_pack(np.ascontiguousarray(comb2.ravel(order="F")), want2, im, jm, km, 1, vd)
        np.testing.assert_array_equal(back.view(np.uint32), want2.view(np.uint32))
        abi.check(L.les_ctx_halo_write(gpu.ctx, h, back.ctypes.data))
        again = gpu.download(NAMES)
        for nm in NAMES:
            np.testing.assert_array_equal(again[nm].view(np.uint32), now[nm].view(np.uint32))
        F = now
    gpu.close()
