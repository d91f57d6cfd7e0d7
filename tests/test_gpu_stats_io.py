"""aveflow (time statistics) on the device and the reference's unformatted
files, against the oracle.

aveflow.f95:42-175 runs after each step on the device-resident state
(les_aveflow) and as a per-routine entry (les_aveflow_); the restart writer
(press.f95:191-201, adam.f95:22-31) and the ICAL=1 reader (ifdata.f95:227-247)
move the state through big-endian gfortran records.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from les_halo_b200 import GpuLes, abi, fields as FL, synthetic_case
from tests.helpers import (assert_bitexact, be_floats, read_fortran_records,
                           write_fortran_records)

pytestmark = pytest.mark.gpu
STATE = FL.STATE + FL.MASKS


def _pair(ip, jp, kp, seed, **kw):
    case = synthetic_case(ip, jp, kp, seed=seed, masks_and_poisson=oracle.masks_and_poisson, **kw)
    return case, case.copy()


def _assert_stats(got, want):
    bad = [n for n in want if not np.array_equal(got[n].view(np.uint32), want[n].view(np.uint32))]
    assert not bad, {n: (int(np.sum(got[n].view(np.uint32) != want[n].view(np.uint32))),
                         float(np.max(np.abs(got[n] - want[n])))) for n in bad}


@pytest.mark.parametrize("dims,n1,nmax", [((24, 20, 16), 2, 6), ((33, 18, 12), 1, 3)])
def test_aveflow_after_each_step(require_gpu, tmp_path, dims, n1, nmax):
    ip, jp, kp = dims
    ref, dev = _pair(ip, jp, kp, seed=31)
    gpu = GpuLes(dev)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    stats = oracle.ave_alloc(ip, jp, kp)
    # uwfxs is intent(inout) and never zeroed by aveflow: start from a value
    stats["uwfxs"][...] = np.random.default_rng(3).standard_normal((ip, kp)).astype(np.float32)
    gpu.aveflow_upload({"uwfxs": stats["uwfxs"].copy(order="F")})
    f10, f11 = tmp_path / "data10", tmp_path / "data11"
    for n in range(1, nmax + 1):
        oracle.run_steps(ref, n, 1)
        gpu.step(n, 1)
        time = np.float32(n - 1) * np.float32(ref.params.dt)  # main_ocl.f95:233
        oracle.aveflow(ref, stats, n, n1, nmax)
        gpu.aveflow(n, n1, nmax, float(time), str(f10) + " " * 8, f11)
    _assert_stats(gpu.aveflow_download(), stats)
    assert_bitexact(gpu.download(STATE), {k: ref.a(k) for k in STATE}, ip, jp, kp, STATE)
    hdr = np.array([nmax], ">i4").tobytes() + np.array([time], ">f4").tobytes()
    r10, r11 = read_fortran_records(f10), read_fortran_records(f11)
    assert r10 == [hdr] + [be_floats(stats[n]) for n in ("aveu", "avew", "avev")]
    assert r11 == [hdr] + [be_floats(stats[n]) for n in ("aveuu", "aveww", "avevv", "uwfx")]
    gpu.close()


def test_aveflow_routine_entry(require_gpu, tmp_path):
    ip, jp, kp = 21, 14, 9
    rng = np.random.default_rng(8)
    case, _ = _pair(ip, jp, kp, seed=5)
    for name in ("u", "v", "w", "p", "sm"):
        a = case.a(name)
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
    stats = oracle.ave_alloc(ip, jp, kp)
    for a in stats.values():
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
    I = lambda x: C.byref(C.c_int(x))

    def call(st, n, n1, nmax, d10=None):
        args = [I(n), I(n1), I(kp), I(jp), I(ip)]
        args += [FL.ptr(st[k]) for k in oracle.AVE_CELL] + [FL.ptr(st[k]) for k in oracle.AVE_COL[:6]]
        args += [FL.ptr(case.a(k)) for k in ("u", "v", "w", "p", "sm")]
        args += [I(nmax), FL.ptr(st["uwfxs"]), d10, C.byref(C.c_float(2.5)), None]
        abi.check(abi.lib().les_aveflow_(*args))

    # accumulate only (n1 < n < nmax), then restart + finish in one call (n == n1 == nmax)
    for n, n1, nmax in ((4, 2, 9), (3, 3, 3), (5, 7, 5)):
        want = {k: v.copy(order="F") for k, v in stats.items()}
        got = {k: v.copy(order="F") for k, v in stats.items()}
        oracle.aveflow(case, want, n, n1, nmax)
        call(got, n, n1, nmax)
        _assert_stats(got, want)
        stats = want
    # file names arrive blank-padded (CHARACTER(len=70))
    d10 = tmp_path / "ave10"
    got = {k: v.copy(order="F") for k, v in stats.items()}
    call(got, 6, 6, 6, str(d10).ljust(70).encode())
    assert len(read_fortran_records(d10)) == 4


def test_restart_write_read_and_resume(require_gpu, tmp_path):
    ip, jp, kp = 24, 16, 12
    ref, dev = _pair(ip, jp, kp, seed=17)
    gpu = GpuLes(dev)
    oracle.ifdata(ref, 1)
    gpu.warmup(1)
    for n in (1, 2, 3):
        oracle.run_steps(ref, n, 1)
        gpu.step(n, 1)
    d20, d21 = tmp_path / "data20", tmp_path / "data21"
    fghold = np.random.default_rng(4).standard_normal((ip, jp, kp)).astype(np.float32)
    fghold = np.asfortranarray(fghold)
    gpu.write_restart(d20, d21, fghold)
    names20 = ["u", "v", "w", "p", "usum", "vsum", "wsum"]
    names21 = ["fold", "gold", "hold"]
    interior = lambda n: FL.interior(n, ref.a(n), ip, jp, kp)
    assert read_fortran_records(d20) == [be_floats(interior(n)) for n in names20]
    assert read_fortran_records(d21) == [be_floats(interior(n)) for n in names21] + [be_floats(fghold)]
    gpu.write_restart(None, d21)  # the OpenCL driver's three-record data21
    assert len(read_fortran_records(d21)) == 3
    gpu.write_restart(None, d21, fghold)

    # ICAL=1 start of a fresh context: data30 = (n,time) + the data20 records
    d30 = tmp_path / "data30"
    hdr = np.array([3], ">i4").tobytes() + np.array([0.1], ">f4").tobytes()
    write_fortran_records(d30, [hdr] + read_fortran_records(d20))
    ref2, dev2 = _pair(ip, jp, kp, seed=17)
    g2 = GpuLes(dev2)
    before = g2.download(STATE)
    fg = np.zeros((ip, jp, kp), np.float32, order="F")
    assert g2.read_restart(d30, d21, fg) == (3, np.float32(0.1))
    assert np.array_equal(fg, fghold)
    after = g2.download(STATE)
    for n in names20 + names21:
        want = before[n].copy(order="F")
        FL.set_interior(n, want, interior(n), ip, jp, kp)  # ghosts kept, interior replaced
        assert_bitexact({n: after[n]}, {n: want}, ip, jp, kp, [n])
    # ... then ifdata's warm-up and steps on both sides
    for n in names20 + names21:
        FL.set_interior(n, ref2.a(n), interior(n), ip, jp, kp)
    oracle.ifdata(ref2, 4)
    g2.warmup(4)
    for n in (4, 5):
        oracle.run_steps(ref2, n, 1)
        g2.step(n, 1)
    assert_bitexact(g2.download(STATE), {k: ref2.a(k) for k in STATE}, ip, jp, kp, STATE)
    g2.close()
    gpu.close()


def test_restart_reader_rejects_bad_files(require_gpu, tmp_path):
    ip, jp, kp = 12, 8, 6
    _, dev = _pair(ip, jp, kp, seed=2)
    g = GpuLes(dev)
    nrec = ip * jp * kp
    good = [np.zeros(nrec, ">f4").tobytes()] * 7
    hdr = np.array([1], ">i4").tobytes() + np.array([0.0], ">f4").tobytes()
    d30, d31 = tmp_path / "d30", tmp_path / "d31"
    write_fortran_records(d31, good[:3])
    L = abi.lib()
    for recs, msg in (([hdr] + good[:6], "record 8 missing"),
                      ([hdr] + good[:6] + [np.zeros(nrec - 1, ">f4").tobytes()], "record 8 holds"),
                      ([hdr[:4]] + good, "record 1 holds")):
        write_fortran_records(d30, recs)
        st = L.les_read_restart(g.ctx, str(d30).encode(), str(d31).encode(), None, None, None)
        assert st == abi.LES_ERR_IO and msg in L.les_last_error_string().decode()
    write_fortran_records(d30, [hdr] + good)
    st = L.les_read_restart(g.ctx, str(d30).encode(), str(d31).encode(), None, None,
                            np.zeros(nrec, np.float32).ctypes.data)
    assert st == abi.LES_ERR_IO and "fghold" in L.les_last_error_string().decode()
    assert L.les_read_restart(g.ctx, str(d30).encode(), str(d31).encode(), None, None, None) == abi.LES_OK
    g.close()


def test_netcdf_from_the_device_state(require_gpu, tmp_path):
    from scipy.io import netcdf_file
    ip, jp, kp = 20, 14, 9
    _, dev = _pair(ip, jp, kp, seed=12)
    g = GpuLes(dev)
    g.warmup(1)
    g.step(1, 2)
    L = abi.lib()
    h = C.c_void_p()
    abi.check(L.les_netcdf_open(f"{tmp_path}/".encode(), ip, jp, kp, 3, C.byref(h)))
    abi.check(L.les_netcdf_write(h, g.ctx, 2))
    abi.check(L.les_netcdf_close(h))
    st = g.download(["p", "u", "w", "usum"])
    for fname, var, src in (("LES_output_p.nc", "pressure", "p"), ("LES_output_u.nc", "velocity_x", "u"),
                            ("LES_output_w.nc", "velocity_z", "w"), ("LES_output_uvwsum.nc", "velocity_sum_x", "usum")):
        with netcdf_file(str(tmp_path / fname), "r", mmap=False) as f:
            assert np.array_equal(f.variables[var][1].copy(), st[src].T)
    g.close()
