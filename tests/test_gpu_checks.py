"""Input checks of the context API: non-finite inputs are refused with
LES_ERR_NAN before anything reaches the device (the reference has no such
check; set.f95:84-88 and ifdata.f95:216-219 are its only hard stops, tested
as LES_ERR_BAD_ARG / LES_ERR_DIMS elsewhere)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from les_halo_b200 import GpuLes, abi, fields as FL, synthetic_case

pytestmark = pytest.mark.gpu


def _case():
    return synthetic_case(24, 20, 16, seed=3, masks_and_poisson=oracle.masks_and_poisson)


@pytest.mark.parametrize("name,idx,val", [("u", (5, 7, 3), np.nan), ("p", (0, 0, 0), np.inf),
                                          ("sm", (-1, -1, 17), -np.inf), ("dzn", (3,), np.nan),
                                          ("wind_profile", (20, 16), np.nan)])
def test_upload_refuses_non_finite(require_gpu, name, idx, val):
    case = _case()
    a = case.a(name)
    a[FL.index(name, case.ip, case.jp, case.kp, *idx)] = val
    p = case.params
    ctx = C.c_void_p()
    abi.check(abi.lib().les_ctx_create(C.byref(p), C.byref(ctx)))
    hf = case.host_fields()
    st = abi.lib().les_ctx_upload(ctx, C.byref(hf))
    msg = abi.lib().les_last_error_string().decode()
    abi.lib().les_ctx_destroy(ctx)
    assert st == abi.LES_ERR_NAN, (st, msg)
    assert name in msg
    if len(idx) == 3:
        assert "(%d,%d,%d)" % idx in msg


def test_set_wind_profile_refuses_non_finite(require_gpu):
    case = _case()
    g = GpuLes(case)
    wp = case.a("wind_profile").copy(order="F")
    g.set_wind_profile(wp)
    wp[3, 4] = np.nan
    with pytest.raises(abi.LesError) as e:
        g.set_wind_profile(wp)
    assert e.value.status == abi.LES_ERR_NAN
    g.close()
