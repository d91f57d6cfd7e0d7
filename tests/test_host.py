"""Host-side logic of the product library (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from les_halo_b200 import abi, fields as FL, synth_cfg

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(les_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


@pytest.mark.parametrize("path", [abi.LIB_PATH, abi.CHECKED_LIB_PATH], ids=["plain", "checked"])
def test_every_declared_symbol_is_exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = sorted(_declared() - exported)
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_library_loads_and_binds():
    lib = abi.lib()  # loads and binds every prototype
    assert lib.les_version().startswith(b"lesb200")


def test_bounds_violations_needs_the_checked_build():
    """The plain library answers les_bounds_violations with LES_ERR_STATE
    (no GPU call is made)."""
    if abi.LIB_PATH != abi.CHECKED_LIB_PATH:
        n = C.c_ulonglong(7)
        assert abi.lib().les_bounds_violations(C.byref(n), None) == abi.LES_ERR_STATE


def test_grid_metrics_match_oracle():
    for ip, jp, kp in [(150, 150, 90), (17, 9, 30)]:
        a = {n: FL.alloc(n, ip, jp, kp) for n in FL.METRICS}
        b = {n: FL.alloc(n, ip, jp, kp) for n in FL.METRICS}
        rng = np.random.default_rng(ip)
        for d in (a, b):
            d["dx1"][:] = np.float32(3.5)
            d["dy1"][:] = np.float32(4.25)
            d["dzn"][2: kp + 3] = (1.0 + rng.random(kp + 1)).astype(np.float32)  # dzn(1..kp+1)
            rng = np.random.default_rng(ip)
        order = ("dx1", "dxl", "dy1", "dyl", "z2", "dzn", "dzs", "dxs", "dys")
        abi.check(abi.lib().les_grid_metrics(ip, jp, kp, *[FL.ptr(a[n]) for n in order]))
        oracle.lib().oracle_grid_metrics(ip, jp, kp, *[FL.ptr(b[n]) for n in order])
        for n in order:
            np.testing.assert_array_equal(a[n], b[n], err_msg=n)


def test_synthetic_inputs_deterministic_and_in_range():
    L = abi.lib()
    cfg = synth_cfg(150, 150, 90, seed=11)
    z1 = FL.alloc("zbm", 150, 150, 90)
    z2 = FL.alloc("zbm", 150, 150, 90)
    f1 = L.les_synth_terrain(C.byref(cfg), FL.ptr(z1))
    f2 = L.les_synth_terrain(C.byref(cfg), FL.ptr(z2))
    assert f1 == f2 and np.array_equal(z1, z2)
    assert 0.30 <= f1 <= 0.34
    built = z1[z1 > 0]
    assert built.min() >= 4.0 and built.max() <= 80.0
    assert 12.0 < float(np.mean(built)) < 30.0


def test_synthetic_inflow_is_log_law():
    ip, jp, kp = 20, 16, 30
    cfg = synth_cfg(ip, jp, kp, seed=2)
    A = {n: FL.alloc(n, ip, jp, kp) for n in FL.METRICS}
    abi.check(abi.lib().les_synth_grid(C.byref(cfg), *[FL.ptr(A[n]) for n in
                                                       ("dx1", "dxl", "dy1", "dyl", "z2", "dzn",
                                                        "dzs", "dxs", "dys")]))
    wp = FL.alloc("wind_profile", ip, jp, kp)
    abi.check(abi.lib().les_synth_inflow(C.byref(cfg), FL.ptr(A["z2"]), FL.ptr(A["dzn"]),
                                         FL.ptr(wp)))
    zc = A["z2"][:kp] + np.float32(0.5) * A["dzn"][2: kp + 2]
    base = (0.3 / 0.4) * np.log(zc.astype(np.float64) / np.float64(np.float32(0.1)))
    ratio = wp / base[None, :]
    assert np.all(np.abs(ratio - 1.0) <= 0.0201)
    assert A["dzn"][2] == np.float32(2.0) and A["dzn"][3] == np.float32(2.0) * np.float32(1.05)


def test_halo_buffer_sizes_match_oracle():
    for (im, jm, km, hw, vd) in [(20, 20, 2, 3, 2), (152, 153, 92, 1, 4), (7, 9, 3, 1, 16)]:
        for inner in (0, 1):
            assert abi.lib().les_halo_buffer_floats(im, jm, km, hw, vd, inner) == \
                oracle.halo_buffer_floats(im, jm, km, hw, vd, bool(inner))


def test_param_validation_needs_no_gpu():
    L = abi.lib()
    p = abi.LesParams()
    abi.check(L.les_params_default(C.byref(p), 16, 12, 40))
    ctx = C.c_void_p()
    # power-law inflow writes k=1..78 (bondv1.f95:26): needs kp >= 78
    assert L.les_ctx_create(C.byref(p), C.byref(ctx)) == abi.LES_ERR_DIMS
    assert b"78" in L.les_last_error_string()
    p.inflow_mode = abi.LES_INFLOW_EXTERNAL
    p.dt = 1.0  # beyond the IBM bound of set.f95:84
    assert L.les_ctx_create(C.byref(p), C.byref(ctx)) == abi.LES_ERR_BAD_ARG
    assert L.les_halo_pack(None, None, 4, 4, 1, 1, 3, 0, None) == abi.LES_ERR_BAD_ARG


def test_field_bounds_table():
    assert FL.bounds("w", 10, 8, 6) == [(0, 11), (-1, 9), (-1, 7)]
    assert FL.bounds("diu1", 10, 8, 6) == [(-1, 12), (0, 10), (0, 8)]
    assert FL.alloc("sm", 10, 8, 6).shape == (13, 11, 8)


@pytest.mark.parametrize("dims,over", [((48, 40, 30), {}), ((60, 44, 20), {"plan_area": 0.35, "h_max": 120.0}),
                                       ((32, 24, 80), {"dx": 3.0, "dy": 5.0})])
def test_oracle_builds_the_library_case(dims, over):
    # CPU-only runs (bench.py's reference arm and CPU baseline) build their
    # cases with the oracle alone; they must be the library's cases bit for
    # bit, parameters included
    from les_halo_b200 import synthetic_case
    ip, jp, kp = dims
    a = oracle.synthetic_case(ip, jp, kp, seed=3, **over)
    b = synthetic_case(ip, jp, kp, seed=3, masks_and_poisson=oracle.masks_and_poisson, **over)
    assert sorted(a.arrays) == sorted(b.arrays)
    for n in a.arrays:
        assert np.array_equal(a.arrays[n].view(np.uint32), b.arrays[n].view(np.uint32)), n
    for f, _ in abi.LesParams._fields_:
        assert np.float32(getattr(a.params, f)) == np.float32(getattr(b.params, f)), f
    assert a.built_fraction == b.built_fraction
