"""Pin the halo pack/unpack oracle to the reference's own C test programs.

tests/golden/halo_kat.json holds what src/OpenCL/test_halo_*.c print
(generated by tests/golden/make_halo_golden.py).  Those programs use a
component-major (SoA) array, which the oracle expresses through its
element/component strides.
"""
import json
from pathlib import Path

import numpy as np

import oracle

KAT = json.loads((Path(__file__).parent / "golden" / "halo_kat.json").read_text())


def _halves(im, jm, km, vdim):
    a = np.empty(vdim * im * jm * km, np.float32)
    a[: a.size // 2] = 1.0
    a[a.size // 2:] = 2.0
    return a


def test_write_standard_kat():
    # test_halo_write.c: array 1/2 halves, buffer all 5, exchange_2_halo_write
    p = KAT["test_halo_write"]["params"]
    im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
    arr = _halves(im, jm, km, vd)
    buf = np.full(vd * 2 * (im + jm - 2 * hw) * hw * km, 5.0, np.float32)
    oracle.halo_unpack(arr, buf, im, jm, km, hw, vd, soa=True)
    np.testing.assert_array_equal(arr, np.array(KAT["test_halo_write"]["printed"], np.float32))


def test_write_correct_kat():
    # test_halo_write_correct.c: same harness, halo_exchange_correct.cl write
    p = KAT["test_halo_write_correct"]["params"]
    im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
    arr = _halves(im, jm, km, vd)
    buf = np.full(vd * 2 * (im + jm - 2 * hw) * hw * km, 5.0, np.float32)
    oracle.halo_unpack(arr, buf, im, jm, km, hw, vd, soa=True, inner=True)
    np.testing.assert_array_equal(arr, np.array(KAT["test_halo_write_correct"]["printed"], np.float32))


def test_read_correct_kat():
    # test_halo_read_correct.c: array[i] = i, buffer -1, inner-ring read;
    # prints the (unchanged) array, then the buffer.
    p = KAT["test_halo_read_correct"]["params"]
    im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
    arr = np.arange(vd * im * jm * km, dtype=np.float32)
    nbuf = vd * 2 * (im + jm - 4 * hw) * hw * km
    assert nbuf == oracle.halo_buffer_floats(im, jm, km, hw, vd, inner=True)
    buf = np.full(nbuf, -1.0, np.float32)
    oracle.halo_pack(arr, buf, im, jm, km, hw, vd, soa=True, inner=True)
    printed = np.array(KAT["test_halo_read_correct"]["printed"], np.float32)
    np.testing.assert_array_equal(printed[: arr.size], arr)
    np.testing.assert_array_equal(printed[arr.size:], buf)


def _testprog_write_variant(arr, buf, im, jm, km, hw, vd):
    """test_halo_read.c's own write (its west/east buffer index is
    `i-h_w+w`, test_halo_read.c:37,39), used only to set up the state its
    read is then applied to."""
    vsz = 2 * km * im * hw + 2 * km * (jm - 2 * hw) * hw
    asz = im * jm * km
    for gl in range(km * max(im, jm)):
        k, i = gl % km, gl // km
        for v in range(vd):
            for w in range(hw):
                if i < im and k < km:
                    arr[i + im * w + k * im * jm + v * asz] = buf[v * vsz + i + im * w + k * im * hw]
                    arr[i + im * w + k * im * jm + im * (jm - hw) + v * asz] = \
                        buf[v * vsz + km * im * hw + i + im * w + k * im * hw]
                if hw - 1 < i < jm - hw and k < km:
                    arr[i * im + w + k * im * jm + v * asz] = \
                        buf[v * vsz + km * im * hw * 2 + i - hw + w + k * (jm - 2 * hw) * hw]
                    arr[i * im + w + k * im * jm + im - hw + v * asz] = \
                        buf[v * vsz + km * im * hw * 2 + km * (jm - 2 * hw) * hw + i - hw + w +
                            k * (jm - 2 * hw) * hw]


def test_read_standard_kat():
    # test_halo_read.c: halves array, buffer sections 6|7|8|9, its write,
    # buffer reset to 4, then exchange_2_halo_read (the restated one).
    p = KAT["test_halo_read"]["params"]
    im, jm, km, hw, vd = p["im"], p["jm"], p["km"], p["h_w"], p["v_dim"]
    arr = _halves(im, jm, km, vd)
    vsz = 2 * km * im * hw + 2 * km * (jm - 2 * hw) * hw
    ns, we = im * hw * km, (jm - 2 * hw) * hw * km
    buf = np.zeros(vd * vsz, np.float32)
    for v in range(vd):
        buf[v * vsz: v * vsz + ns] = 6
        buf[v * vsz + ns: v * vsz + 2 * ns] = 7
        buf[v * vsz + 2 * ns: v * vsz + 2 * ns + we] = 8
        buf[v * vsz + 2 * ns + we: v * vsz + 2 * ns + 2 * we] = 9
    _testprog_write_variant(arr, buf, im, jm, km, hw, vd)
    buf[:] = 4.0
    oracle.halo_pack(arr, buf, im, jm, km, hw, vd, soa=True)
    np.testing.assert_array_equal(buf, np.array(KAT["test_halo_read"]["printed"], np.float32))
