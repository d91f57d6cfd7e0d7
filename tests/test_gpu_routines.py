"""Per-routine drop-in entries (Fortran argument order) against the oracle.

Inputs come from a synthetic case advanced two steps by the oracle.  Output
arrays are pre-filled with garbage so that elements a reference routine
never writes must come back unchanged, as they would from the Fortran.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from les_halo_b200 import abi, fields as FL, synthetic_case
from tests.helpers import assert_bitexact

pytestmark = pytest.mark.gpu
IP, JP, KP = 21, 14, 11
P = C.c_void_p
I = lambda x: C.byref(C.c_int(x))
Fv = lambda x: C.byref(C.c_float(x))


@pytest.fixture(scope="module")
def state():
    case = synthetic_case(IP, JP, KP, seed=13, masks_and_poisson=oracle.masks_and_poisson)
    oracle.ifdata(case, 1)
    oracle.run_steps(case, 1, 2)
    return case


def _ol():
    L = oracle.lib()
    i, f, p = C.c_int, C.c_float, P
    L.oracle_velnw.argtypes = [i, i, i, p, f, p, p, f, p, p, p, p, p, p, p]
    L.oracle_bondv1.argtypes = [i, p, p, p, p, p, i, i, i, f, p]
    L.oracle_bondv1_ext_wind_profile.argtypes = [i, p, p, p, p, p, i, i, i, f, p, p]
    L.oracle_velfg.argtypes = [i, i, i, p, p, p, p, p, p, p, p, p, p, f] + [p] * 30
    L.oracle_feedbf.argtypes = [i, i, i] + [p] * 9 + [f, f, f] + [p] * 6
    L.oracle_les.argtypes = [i, p, p, p, p, i, i] + [p] * 13
    L.oracle_boundsm.argtypes = [i, i, p, i]
    L.oracle_adam.argtypes = [i, i, p, i, i, i, p, p, p, p, p]
    L.oracle_bondfg.argtypes = [i, i, p, i, p, p]
    L.oracle_boundp1.argtypes = [i, i, p, i]
    L.oracle_boundp2.argtypes = [i, i, p, i]
    L.oracle_press.argtypes = [i, i, i, p, p, p, p, p, p, p, p, p, p, f, p, p, p, p, p, p, p, p, i, i,
                               p, p, p]
    L.oracle_press.restype = C.c_int
    return L


def _cp(d):
    return {k: v.copy(order="F") for k, v in d.items()}


def _garbage(name, seed):
    a = FL.alloc(name, IP, JP, KP)
    a[...] = np.random.default_rng(seed).standard_normal(a.shape).astype(np.float32)
    return a


def test_velnw(require_gpu, state):
    A = state.arrays
    names = ["p", "u", "v", "w", "f", "g", "h", "dxs", "dys", "dzs"]
    a, b = _cp({n: A[n] for n in names}), _cp({n: A[n] for n in names})
    ro, dt = state.params.ro, state.params.dt
    _ol().oracle_velnw(KP, JP, IP, FL.ptr(a["p"]), ro, FL.ptr(a["dxs"]), FL.ptr(a["u"]), dt,
                       FL.ptr(a["f"]), FL.ptr(a["dys"]), FL.ptr(a["v"]), FL.ptr(a["g"]),
                       FL.ptr(a["dzs"]), FL.ptr(a["w"]), FL.ptr(a["h"]))
    abi.check(abi.lib().les_velnw_(I(KP), I(JP), I(IP), FL.ptr(b["p"]), Fv(ro), FL.ptr(b["dxs"]),
                                   FL.ptr(b["u"]), Fv(dt), FL.ptr(b["f"]), FL.ptr(b["dys"]),
                                   FL.ptr(b["v"]), FL.ptr(b["g"]), FL.ptr(b["dzs"]), FL.ptr(b["w"]),
                                   FL.ptr(b["h"])))
    assert_bitexact(b, a, IP, JP, KP, ["u", "v", "w"])


@pytest.mark.parametrize("n", [1, 7])
def test_bondv1_ext(require_gpu, state, n):
    A = state.arrays
    names = ["u", "v", "w", "z2", "dzn", "dxs", "wind_profile"]
    a, b = _cp({k: A[k] for k in names}), _cp({k: A[k] for k in names})
    dt = state.params.dt
    _ol().oracle_bondv1_ext_wind_profile(JP, FL.ptr(a["u"]), FL.ptr(a["z2"]), FL.ptr(a["dzn"]),
                                         FL.ptr(a["v"]), FL.ptr(a["w"]), KP, n, IP, dt,
                                         FL.ptr(a["dxs"]), FL.ptr(a["wind_profile"]))
    abi.check(abi.lib().les_bondv1_ext_wind_profile_(
        I(JP), FL.ptr(b["u"]), FL.ptr(b["z2"]), FL.ptr(b["dzn"]), FL.ptr(b["v"]), FL.ptr(b["w"]),
        I(KP), I(n), I(IP), Fv(dt), FL.ptr(b["dxs"]), FL.ptr(b["wind_profile"])))
    assert_bitexact(b, a, IP, JP, KP, ["u", "v", "w"])


def test_bondv1_power_law(require_gpu):
    ip, jp, kp = 9, 6, 80
    case = synthetic_case(ip, jp, kp, seed=2, inflow="power",
                          masks_and_poisson=oracle.masks_and_poisson)
    A = case.arrays
    rng = np.random.default_rng(1)
    for n in ("u", "v", "w"):
        A[n][...] = rng.standard_normal(A[n].shape).astype(np.float32)
    a, b = _cp(A), _cp(A)
    dt = case.params.dt
    _ol().oracle_bondv1(jp, FL.ptr(a["u"]), FL.ptr(a["z2"]), FL.ptr(a["dzn"]), FL.ptr(a["v"]),
                        FL.ptr(a["w"]), kp, 3, ip, dt, FL.ptr(a["dxs"]))
    abi.check(abi.lib().les_bondv1_(I(jp), FL.ptr(b["u"]), FL.ptr(b["z2"]), FL.ptr(b["dzn"]),
                                    FL.ptr(b["v"]), FL.ptr(b["w"]), I(kp), I(3), I(ip), Fv(dt),
                                    FL.ptr(b["dxs"])))
    assert_bitexact(b, a, ip, jp, kp, ["u", "v", "w"])
    # km < 78 is out of the power law's range (bondv1.f95:26)
    assert abi.lib().les_bondv1_(I(6), FL.ptr(b["u"]), FL.ptr(b["z2"]), FL.ptr(b["dzn"]),
                                 FL.ptr(b["v"]), FL.ptr(b["w"]), I(40), I(3), I(9), Fv(dt),
                                 FL.ptr(b["dxs"])) == abi.LES_ERR_DIMS


VEL2 = ([f"cov{n}" for n in range(1, 4)] + ["dfu1"] + [f"diu{n}" for n in (1, 2)] + ["dy1"] +
        ["diu3", "dzn", "vn", "f"] + [f"cov{n}" for n in (4, 5, 6)] + ["dfv1"] +
        [f"diu{n}" for n in (4, 5, 6)] + ["g"] + [f"cov{n}" for n in (7, 8, 9)] + ["dfw1"] +
        [f"diu{n}" for n in (7, 8, 9)] + ["dzs", "h", "nou1", "u", "nou5", "v", "nou9", "w"] +
        [f"nou{n}" for n in (2, 3, 4, 6, 7, 8)])


def _velfg_arrays(state):
    A = state.arrays
    d = {}
    for n in VEL2:
        if n == "vn":
            continue
        if n in A:
            d[n] = A[n].copy(order="F")
        else:
            d[n] = _garbage(n, hash(n) % 1000)
    d["dx1"] = A["dx1"].copy(order="F")
    return d


def test_velfg_all_outputs(require_gpu, state):
    a, b = _velfg_arrays(state), _velfg_arrays(state)
    vn = state.params.vn
    args_o = [KP, JP, IP, FL.ptr(a["dx1"])] + [vn if n == "vn" else FL.ptr(a[n]) for n in VEL2]
    _ol().oracle_velfg(*args_o)
    args_p = [I(KP), I(JP), I(IP), FL.ptr(b["dx1"])] + [Fv(vn) if n == "vn" else FL.ptr(b[n])
                                                        for n in VEL2]
    abi.check(abi.lib().les_velfg_(*args_p))
    outs = [n for n in VEL2 if n not in ("vn", "dy1", "dzn", "dzs", "u", "v", "w")]
    assert_bitexact(b, a, IP, JP, KP, outs)


def test_velfg_null_scratch(require_gpu, state):
    a, b = _velfg_arrays(state), _velfg_arrays(state)
    vn = state.params.vn
    _ol().oracle_velfg(*([KP, JP, IP, FL.ptr(a["dx1"])] +
                         [vn if n == "vn" else FL.ptr(a[n]) for n in VEL2]))
    keep = {"dy1", "dzn", "dzs", "u", "v", "w", "f", "g", "h"} | {f"diu{n}" for n in range(1, 10)}
    args_p = [I(KP), I(JP), I(IP), FL.ptr(b["dx1"])] + [
        Fv(vn) if n == "vn" else (FL.ptr(b[n]) if n in keep else None) for n in VEL2]
    abi.check(abi.lib().les_velfg_(*args_p))
    assert_bitexact(b, a, IP, JP, KP, ["f", "g", "h"] + [f"diu{n}" for n in range(1, 10)])


def test_feedbf(require_gpu, state):
    A = state.arrays
    names = ["usum", "u", "bmask1", "vsum", "v", "cmask1", "wsum", "w", "dmask1"]
    base = {n: A[n] for n in names}
    base.update({n: _garbage(n, i) for i, n in enumerate(("fx", "fy", "fz"))})
    base.update({n: A[n] for n in ("f", "g", "h")})
    a, b = _cp(base), _cp(base)
    p = state.params
    order = names + ["fx", "fy", "fz", "f", "g", "h"]
    _ol().oracle_feedbf(KP, JP, IP, *[FL.ptr(a[n]) for n in names], p.alpha, p.dt, p.beta,
                        *[FL.ptr(a[n]) for n in order[9:]])
    abi.check(abi.lib().les_feedbf_(I(KP), I(JP), I(IP), *[FL.ptr(b[n]) for n in names], Fv(p.alpha),
                                    Fv(p.dt), Fv(p.beta), *[FL.ptr(b[n]) for n in order[9:]]))
    assert_bitexact(b, a, IP, JP, KP, ["usum", "vsum", "wsum", "fx", "fy", "fz", "f", "g", "h"])


def test_les_from_caller_diu(require_gpu, state):
    # diu arrays from velfg with garbage wherever vel2 never writes
    d = _velfg_arrays(state)
    _ol().oracle_velfg(*([KP, JP, IP, FL.ptr(d["dx1"])] +
                         [state.params.vn if n == "vn" else FL.ptr(d[n]) for n in VEL2]))
    A = state.arrays
    base = {f"diu{n}": d[f"diu{n}"] for n in range(1, 10)}
    base.update({n: A[n] for n in ("dx1", "dy1", "dzn", "f", "g", "h")})
    base["sm"] = _garbage("sm", 77)
    base["delx1"] = FL.alloc("delx1", IP, JP, KP)
    a, b = _cp(base), _cp(base)
    diu = [f"diu{n}" for n in range(1, 10)]
    _ol().oracle_les(KP, FL.ptr(a["delx1"]), FL.ptr(a["dx1"]), FL.ptr(a["dy1"]), FL.ptr(a["dzn"]), JP,
                     IP, *[FL.ptr(a[n]) for n in diu], FL.ptr(a["sm"]), FL.ptr(a["f"]), FL.ptr(a["g"]),
                     FL.ptr(a["h"]))
    abi.check(abi.lib().les_les_(I(KP), FL.ptr(b["delx1"]), FL.ptr(b["dx1"]), FL.ptr(b["dy1"]),
                                 FL.ptr(b["dzn"]), I(JP), I(IP), *[FL.ptr(b[n]) for n in diu],
                                 FL.ptr(b["sm"]), FL.ptr(b["f"]), FL.ptr(b["g"]), FL.ptr(b["h"])))
    assert_bitexact(b, a, IP, JP, KP, ["sm", "f", "g", "h", "delx1"])


def test_boundsm_adam_bondfg_boundp(require_gpu, state):
    A = state.arrays
    L, O = abi.lib(), _ol()
    a, b = {"sm": _garbage("sm", 5)}, None
    b = _cp(a)
    O.oracle_boundsm(KP, JP, FL.ptr(a["sm"]), IP)
    abi.check(L.les_boundsm_(I(KP), I(JP), FL.ptr(b["sm"]), I(IP)))
    assert_bitexact(b, a, IP, JP, KP, ["sm"])

    base = {n: A[n] for n in ("fold", "gold", "hold", "f", "g", "h")}
    a, b = _cp(base), _cp(base)
    O.oracle_adam(3, 10, FL.ptr(a["fold"]), IP, JP, KP, FL.ptr(a["gold"]), FL.ptr(a["hold"]),
                  FL.ptr(a["f"]), FL.ptr(a["g"]), FL.ptr(a["h"]))
    abi.check(L.les_adam_(I(3), I(10), FL.ptr(b["fold"]), I(IP), I(JP), I(KP), FL.ptr(b["gold"]),
                          FL.ptr(b["hold"]), FL.ptr(b["f"]), FL.ptr(b["g"]), FL.ptr(b["h"])))
    assert_bitexact(b, a, IP, JP, KP, list(base))

    base = {n: _garbage(n, i) for i, n in enumerate(("f", "g", "h"))}
    a, b = _cp(base), _cp(base)
    O.oracle_bondfg(KP, JP, FL.ptr(a["f"]), IP, FL.ptr(a["g"]), FL.ptr(a["h"]))
    abi.check(L.les_bondfg_(I(KP), I(JP), FL.ptr(b["f"]), I(IP), FL.ptr(b["g"]), FL.ptr(b["h"])))
    assert_bitexact(b, a, IP, JP, KP, list(base))

    for fn_o, fn_p, args in ((O.oracle_boundp1, L.les_boundp1_, "kjpi"),
                             (O.oracle_boundp2, L.les_boundp2_, "jipk")):
        a = {"p": _garbage("p", 9)}
        b = _cp(a)
        val = {"k": KP, "j": JP, "i": IP}
        fn_o(*[FL.ptr(a["p"]) if ch == "p" else val[ch] for ch in args])
        abi.check(fn_p(*[FL.ptr(b["p"]) if ch == "p" else I(val[ch]) for ch in args]))
        assert_bitexact(b, a, IP, JP, KP, ["p"])


def test_press(require_gpu, state):
    A = state.arrays
    names = ["rhs", "u", "dx1", "v", "dy1", "w", "dzn", "f", "g", "h", "cn1", "cn2l", "p", "cn2s",
             "cn3l", "cn3s", "cn4l", "cn4s"]
    base = {n: A[n] for n in names}
    base["rhs"] = _garbage("rhs", 3)
    a, b = _cp(base), _cp(base)
    dt = state.params.dt
    o_args = [FL.ptr(a[n]) for n in names]
    it_o = _ol().oracle_press(KP, JP, IP, *o_args[:10], dt, *o_args[10:], 4, 10, None, None, None)
    it = C.c_int()
    p_args = [FL.ptr(b[n]) for n in names]
    abi.check(abi.lib().les_press_(I(KP), I(JP), I(IP), *p_args[:10], Fv(dt), *p_args[10:], I(4),
                                   I(10), C.byref(it)))
    assert it.value == it_o
    assert_bitexact(b, a, IP, JP, KP, ["rhs", "p", "f", "g", "h"])


# ---- press.f95 sub-steps ---------------------------------------------------

def _press_ex():
    return oracle.lib().oracle_press_ex  # signature bound in oracle/__init__.py


_PRESS = ["rhs", "u", "dx1", "v", "dy1", "w", "dzn", "f", "g", "h", "cn1", "cn2l", "p", "cn2s",
          "cn3l", "cn3s", "cn4l", "cn4s"]


def _press_base(state):
    base = {n: state.arrays[n] for n in _PRESS}
    base["rhs"] = _garbage("rhs", 5)
    return _cp(base)


def _oracle_press(a, dt, nmaxp):
    sor, rhsav, pav = C.c_float(), C.c_float(), C.c_float()
    args = [FL.ptr(a[n]) for n in _PRESS]
    _press_ex()(KP, JP, IP, *args[:10], dt, *args[10:], nmaxp, -1.0, 1.0, C.byref(sor), C.byref(rhsav),
                C.byref(pav))
    return sor.value, rhsav.value, pav.value


def _bits(x):
    return np.float32(x).view(np.uint32)


def test_press_rhsav_and_pav_adj(require_gpu, state):
    dt = state.params.dt
    a, b = _press_base(state), _press_base(state)
    _, rhsav_o, pav_o = _oracle_press(a, dt, 0)
    L = abi.lib()
    rhsav, pav = C.c_float(), C.c_float()
    abi.check(L.les_press_rhsav_(I(KP), I(JP), I(IP), *[FL.ptr(b[n]) for n in _PRESS[:10]], Fv(dt),
                                 C.byref(rhsav)))
    assert _bits(rhsav.value) == _bits(rhsav_o)
    abi.check(L.les_press_pav_adj_(I(KP), I(JP), I(IP), FL.ptr(b["p"]), FL.ptr(b["dx1"]), FL.ptr(b["dy1"]),
                                   FL.ptr(b["dzn"]), C.byref(pav)))
    assert _bits(pav.value) == _bits(pav_o)
    assert_bitexact(b, a, IP, JP, KP, ["rhs", "f", "g", "h", "p"])


def test_press_sub_steps_compose_one_iteration(require_gpu, state):
    dt = state.params.dt
    a, b = _press_base(state), _press_base(state)
    sor_o, _, _ = _oracle_press(a, dt, 1)
    L = abi.lib()
    abi.check(L.les_press_rhsav_(I(KP), I(JP), I(IP), *[FL.ptr(b[n]) for n in _PRESS[:10]], Fv(dt), None))
    # two colour sweeps plus boundp2 on a copy must equal the full iteration
    c2 = _cp({"rhs": b["rhs"], "p": b["p"]})
    sor = C.c_float()
    cn = [FL.ptr(b[n]) for n in ("cn1", "cn2l")]
    tail = [FL.ptr(b[n]) for n in ("cn2s", "cn3l", "cn3s", "cn4l", "cn4s")]
    abi.check(L.les_press_residual_(I(KP), I(JP), I(IP), FL.ptr(b["rhs"]), *cn, FL.ptr(b["p"]), *tail,
                                    C.byref(sor)))
    assert _bits(sor.value) == _bits(sor_o)
    for nrd in (0, 1):
        abi.check(L.les_press_sor_sweep_(I(KP), I(JP), I(IP), FL.ptr(c2["rhs"]), *cn, FL.ptr(c2["p"]), *tail,
                                         I(nrd), None))
    abi.check(L.les_boundp2_(I(JP), I(IP), FL.ptr(c2["p"]), I(KP)))
    assert_bitexact({"p": c2["p"]}, {"p": b["p"]}, IP, JP, KP, ["p"])
    abi.check(L.les_press_pav_adj_(I(KP), I(JP), I(IP), FL.ptr(b["p"]), FL.ptr(b["dx1"]), FL.ptr(b["dy1"]),
                                   FL.ptr(b["dzn"]), None))
    assert_bitexact(b, a, IP, JP, KP, ["rhs", "f", "g", "h", "p"])
