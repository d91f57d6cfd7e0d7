"""NetCDF output (module_LES_write_netcdf.f95) written by the library's host
code and read back with scipy's independent NetCDF3 reader (no GPU)."""
import ctypes as C

import numpy as np
import pytest
from scipy.io import netcdf_file

from les_halo_b200 import abi, fields as FL

FILES = {"LES_output.nc": ["pressure"], "LES_output_p.nc": ["pressure"], "LES_output_u.nc": ["velocity_x"],
         "LES_output_v.nc": ["velocity_y"], "LES_output_w.nc": ["velocity_z"],
         "LES_output_uvwsum.nc": ["velocity_sum_x", "velocity_sum_y", "velocity_sum_z"]}
SRC = {"pressure": "p", "velocity_x": "u", "velocity_y": "v", "velocity_z": "w", "velocity_sum_x": "usum",
       "velocity_sum_y": "vsum", "velocity_sum_z": "wsum"}
FILL = np.float32(9.9692099683868690e+36)


def _arrays(ip, jp, kp, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for n in ("p", "u", "v", "w", "usum", "vsum", "wsum"):
        a = FL.alloc(n, ip, jp, kp)
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
        out[n] = a
    return out


def _write(h, t, a):
    L = abi.lib()
    abi.check(L.les_netcdf_write_host(h, t, *[FL.ptr(a[n]) for n in ("p", "u", "v", "w", "usum", "vsum", "wsum")]))


@pytest.mark.parametrize("dims,version", [((7, 5, 4), 1), ((12, 9, 6), 1), ((7, 5, 4), 2)])
def test_files_read_back(tmp_path, monkeypatch, dims, version):
    # version 2 (64-bit offsets) is what files of 2 GiB and more get; forced here
    if version == 2:
        monkeypatch.setenv("LES_NETCDF_64BIT", "1")
    ip, jp, kp = dims
    L = abi.lib()
    h = C.c_void_p()
    abi.check(L.les_netcdf_open(f"{tmp_path}/".encode(), ip, jp, kp, 4, C.byref(h)))
    a1, a3 = _arrays(ip, jp, kp, 1), _arrays(ip, jp, kp, 3)
    _write(h, 1, a1)
    _write(h, 3, a3)
    assert L.les_netcdf_write_host(h, 5, *[FL.ptr(a1[n]) for n in ("p", "u", "v", "w", "usum", "vsum", "wsum")]) \
        == abi.LES_ERR_BAD_ARG  # outside the time dimension
    abi.check(L.les_netcdf_close(h))
    for fname, varnames in FILES.items():
        with netcdf_file(str(tmp_path / fname), "r", mmap=False) as f:
            assert f.version_byte == version
            assert f.dimensions["time"] == 4
            assert list(f.variables["time"][:]) == [1.0, 2.0, 3.0, 4.0]
            assert f.variables["time"].units == b"hours since 2014-08-05 16:00:00"
            assert f.variables["latitude"].units == b"degrees_north"
            assert f.variables["longitude"].units == b"degrees_east"
            for vn in varnames:
                var = f.variables[vn]
                assert var.dimensions == ("time", "level", "latitude", "longitude")
                assert var.units == (b"hPa" if vn == "pressure" else b"m/s")
                src = SRC[vn]
                shape = a1[src].shape  # Fortran (i, j, k) -> file (k, j, i)
                assert var.shape == (4,) + shape[::-1]
                assert f.dimensions["longitude"] == shape[0] and f.dimensions["level"] == shape[2]
                assert np.array_equal(f.variables["latitude"][:], np.arange(1, shape[1] + 1, dtype=np.float32))
                data = var[:].copy()
                assert np.array_equal(data[0], a1[src].T)
                assert np.array_equal(data[2], a3[src].T)
                assert np.all(data[1] == FILL) and np.all(data[3] == FILL)


def test_open_rejects_unwritable_prefix(tmp_path):
    h = C.c_void_p()
    st = abi.lib().les_netcdf_open(f"{tmp_path}/missing/dir/".encode(), 4, 4, 4, 2, C.byref(h))
    assert st == abi.LES_ERR_IO and not h.value
