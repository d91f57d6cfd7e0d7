"""Halo pack/unpack and the setup kernels on the GPU, against the oracle."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from les_halo_b200 import abi, fields as FL, synth_cfg

pytestmark = pytest.mark.gpu
KAT = json.loads((Path(__file__).parent / "golden" / "halo_kat.json").read_text())

CASES = [(20, 20, 2, 3), (7, 9, 3, 1), (13, 11, 5, 2), (152, 153, 4, 1)]


def _gpu_call(fn, a, b, im, jm, km, hw, vd, device):
    L = abi.lib()
    if not device:
        abi.check(getattr(L, fn)(a.ctypes.data, b.ctypes.data, im, jm, km, hw, vd, 0, None))
        return
    import torch
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    abi.check(getattr(L, fn)(ta.data_ptr(), tb.data_ptr(), im, jm, km, hw, vd, 1, None))
    torch.cuda.synchronize()
    a[...] = ta.cpu().numpy()
    b[...] = tb.cpu().numpy()


@pytest.mark.parametrize("vd", [1, 2, 4, 16])
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("device", [0, 1])
def test_pack_unpack_vs_oracle(require_gpu, vd, case, device):
    im, jm, km, hw = case
    rng = np.random.default_rng(im * 1000 + vd)
    for inner in (False, True):
        arr = rng.standard_normal(vd * im * jm * km).astype(np.float32)
        nb = oracle.halo_buffer_floats(im, jm, km, hw, vd, inner)
        b_ref = np.zeros(nb, np.float32)
        b_gpu = np.zeros(nb, np.float32)
        oracle.halo_pack(arr, b_ref, im, jm, km, hw, vd, inner=inner)
        _gpu_call("les_halo_pack_inner" if inner else "les_halo_pack", arr.copy(), b_gpu, im, jm,
                  km, hw, vd, device)
        np.testing.assert_array_equal(b_gpu, b_ref)
        nb_w = oracle.halo_buffer_floats(im, jm, km, hw, vd, False)
        buf = rng.standard_normal(nb_w).astype(np.float32)
        a_ref = arr.copy()
        a_gpu = arr.copy()
        oracle.halo_unpack(a_ref, buf, im, jm, km, hw, vd, inner=inner)
        _gpu_call("les_halo_unpack_inner" if inner else "les_halo_unpack", a_gpu, buf.copy(), im,
                  jm, km, hw, vd, device)
        np.testing.assert_array_equal(a_gpu, a_ref)


def _soa_to_aos(a, vd):
    return np.ascontiguousarray(a.reshape(vd, -1).T).ravel()


def _aos_to_soa(a, vd):
    return np.ascontiguousarray(a.reshape(-1, vd).T).ravel()


def test_reference_kats_through_gpu(require_gpu):
    p = KAT["test_halo_read_correct"]["params"]
    im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
    arr = np.arange(vd * im * jm * km, dtype=np.float32)
    buf = np.full(abi.lib().les_halo_buffer_floats(im, jm, km, hw, vd, 1), -1.0, np.float32)
    aos = _soa_to_aos(arr, vd)  # named: a temporary could be freed before the call reads it
    abi.check(abi.lib().les_halo_pack_inner(aos.ctypes.data, buf.ctypes.data, im, jm, km, hw, vd,
                                            0, None))
    printed = np.array(KAT["test_halo_read_correct"]["printed"], np.float32)
    np.testing.assert_array_equal(buf, printed[arr.size:])
    for prog, fn in (("test_halo_write", "les_halo_unpack"),
                     ("test_halo_write_correct", "les_halo_unpack_inner")):
        p = KAT[prog]["params"]
        im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
        arr = np.empty(vd * im * jm * km, np.float32)
        arr[: arr.size // 2], arr[arr.size // 2:] = 1.0, 2.0
        aos = _soa_to_aos(arr, vd)
        buf = np.full(vd * 2 * (im + jm - 2 * hw) * hw * km, 5.0, np.float32)
        abi.check(getattr(abi.lib(), fn)(aos.ctypes.data, buf.ctypes.data, im, jm, km, hw, vd, 0,
                                         None))
        np.testing.assert_array_equal(_aos_to_soa(aos, vd),
                                      np.array(KAT[prog]["printed"], np.float32))


@pytest.mark.parametrize("dims", [(150, 150, 90), (31, 17, 23)])
def test_masks_and_poisson_bitexact(require_gpu, dims):
    ip, jp, kp = dims
    L = abi.lib()
    cfg = synth_cfg(ip, jp, kp, seed=21)
    A = {n: FL.alloc(n, ip, jp, kp) for n in FL.METRICS}
    abi.check(L.les_synth_grid(C.byref(cfg), *[FL.ptr(A[n]) for n in
                                               ("dx1", "dxl", "dy1", "dyl", "z2", "dzn", "dzs",
                                                "dxs", "dys")]))
    zbm = FL.alloc("zbm", ip, jp, kp)
    L.les_synth_terrain(C.byref(cfg), FL.ptr(zbm))
    g = {n: FL.alloc(n, ip, jp, kp) for n in FL.MASKS + FL.POISSON}
    o = {n: FL.alloc(n, ip, jp, kp) for n in FL.MASKS + FL.POISSON}
    abi.check(L.les_building_masks(ip, jp, kp, FL.ptr(zbm), FL.ptr(A["z2"]), FL.ptr(A["dzn"]),
                                   *[FL.ptr(g[n]) for n in FL.MASKS]))
    abi.check(L.les_poisson_coeffs(ip, jp, kp, FL.ptr(A["dxs"]), FL.ptr(A["dys"]), FL.ptr(A["dzs"]),
                                   *[FL.ptr(g[n]) for n in FL.POISSON]))

    class _C:
        pass
    c = _C()
    c.ip, c.jp, c.kp, c.arrays = ip, jp, kp, dict(A, **o)
    oracle.masks_and_poisson(c, zbm)
    for n in FL.MASKS + FL.POISSON:
        np.testing.assert_array_equal(g[n], o[n], err_msg=n)
    assert g["amask1"].min() == 0.0  # buildings present


@pytest.mark.parametrize("vd", [1, 2, 4, 16])
def test_per_width_entries_match_the_oracle(require_gpu, vd):
    # les_halo_{pack,unpack}[_inner]_<vd> (host pointers)
    im, jm, km, hw = 13, 11, 5, 2
    L = abi.lib()
    rng = np.random.default_rng(vd)
    for inner, sfx in ((False, ""), (True, "_inner")):
        arr = rng.standard_normal(vd * im * jm * km).astype(np.float32)
        nb = oracle.halo_buffer_floats(im, jm, km, hw, vd, inner)
        b_ref = np.zeros(nb, np.float32)
        b_gpu = np.zeros(nb, np.float32)
        oracle.halo_pack(arr, b_ref, im, jm, km, hw, vd, inner=inner)
        abi.check(getattr(L, f"les_halo_pack{sfx}_{vd}")(arr.ctypes.data, b_gpu.ctypes.data, im, jm, km, hw, 0,
                                                         None))
        np.testing.assert_array_equal(b_gpu, b_ref)
        buf = rng.standard_normal(oracle.halo_buffer_floats(im, jm, km, hw, vd, False)).astype(np.float32)
        a_ref, a_gpu = arr.copy(), arr.copy()
        oracle.halo_unpack(a_ref, buf, im, jm, km, hw, vd, inner=inner)
        abi.check(getattr(L, f"les_halo_unpack{sfx}_{vd}")(a_gpu.ctypes.data, buf.ctypes.data, im, jm, km, hw, 0,
                                                           None))
        np.testing.assert_array_equal(a_gpu, a_ref)
