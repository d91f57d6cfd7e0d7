"""Adjoint entries of the linear routines by dot-product tests against the
FP64 oracle.

With its SOR iteration count fixed, press (press.f95:49-146) is a linear map
F from (rhs, u, v, w, f, g, h, p) to (rhs, p, f, g, h), every array over its
full Fortran bounds, with the elements press never touches passed through
(tests/test_press_linear.py checks the linearity on the FP64 oracle); velnw,
feedbf (masks fixed) and adam are linear as written.  For random x and y,
<F x, y> from the FP64 oracle must equal <x, F^T y> with F^T y from the CUDA
adjoint (FP32 arithmetic), to within TOL of sum |x_i (F^T y)_i|.  A wrong
coefficient, index or pass-through breaks the equality by orders of
magnitude more.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import fp64
from les_halo_b200 import abi, fields as FL, synthetic_case

pytestmark = pytest.mark.gpu
IP, JP, KP = 24, 20, 12
TOL = 2e-5
IN = ["rhs", "u", "v", "w", "f", "g", "h", "p"]
OUT = ["rhs", "p", "f", "g", "h"]
COEF = ["dx1", "dy1", "dzn", "cn1", "cn2l", "cn2s", "cn3l", "cn3s", "cn4l", "cn4s"]
I = lambda x: C.byref(C.c_int(x))
Fv = lambda x: C.byref(C.c_float(x))


def press64(case, x, niter):
    """The FP64 oracle's press on float64 copies of x with niter iterations
    (no stop test); returns its outputs."""
    L = fp64.lib()
    i, d, p = C.c_int, C.c_double, C.c_void_p
    L.oracle_press_ex.argtypes = [i, i, i] + [p] * 10 + [d] + [p] * 8 + [i, d, d, p, p, p]
    L.oracle_press_ex.restype = C.c_int
    a = {n: np.asfortranarray(x[n].astype(np.float64)) for n in IN}
    a.update({n: np.asfortranarray(case.arrays[n].astype(np.float64)) for n in COEF})
    P = lambda n: a[n].ctypes.data
    pr = case.params
    it = L.oracle_press_ex(KP, JP, IP, P("rhs"), P("u"), P("dx1"), P("v"), P("dy1"), P("w"), P("dzn"),
                           P("f"), P("g"), P("h"), float(np.float32(pr.dt)), P("cn1"), P("cn2l"), P("p"),
                           P("cn2s"), P("cn3l"), P("cn3s"), P("cn4l"), P("cn4s"), niter, -1.0,
                           float(np.float32(pr.omega)), None, None, None)
    assert it == niter
    return {n: a[n] for n in OUT}


def press_b(case, y, niter):
    """les_press_b_ on copies of the output adjoints y; returns the input adjoints."""
    A = case.arrays
    b = {n: y[n].copy(order="F") for n in OUT}
    for n in ("u", "v", "w"):
        b[n] = FL.alloc(n, IP, JP, KP)
    Fp = FL.ptr
    pr = case.params
    abi.check(abi.lib().les_press_b_(
        I(KP), I(JP), I(IP), Fp(b["rhs"]), Fp(A["dx1"]), Fp(A["dy1"]), Fp(A["dzn"]), Fp(b["f"]), Fp(b["g"]),
        Fp(b["h"]), Fv(pr.dt), Fp(A["cn1"]), Fp(A["cn2l"]), Fp(b["p"]), Fp(A["cn2s"]), Fp(A["cn3l"]),
        Fp(A["cn3s"]), Fp(A["cn4l"]), Fp(A["cn4s"]), I(niter), Fv(pr.omega), Fp(b["u"]), Fp(b["v"]),
        Fp(b["w"])))
    return b


def rand_fields(names, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for n in names:
        a = FL.alloc(n, IP, JP, KP)
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
        out[n] = a
    return out


def check_dot(fx, y, x, g, outs, ins):
    """<F x, y> == <x, F^T y> to TOL of sum |x (F^T y)|."""
    lhs = sum(float(np.sum(fx[n] * y[n].astype(np.float64))) for n in outs)
    terms = [x[n].astype(np.float64) * g[n].astype(np.float64) for n in ins]
    rhs = sum(float(t.sum()) for t in terms)
    scale = sum(float(np.abs(t).sum()) for t in terms)
    assert scale > 0.0
    assert abs(lhs - rhs) <= TOL * scale, (lhs, rhs, scale)


def f64(a):
    return np.asfortranarray(a.astype(np.float64))


@pytest.fixture(scope="module")
def case():
    return synthetic_case(IP, JP, KP, seed=21, masks_and_poisson=oracle.masks_and_poisson)


@pytest.mark.parametrize("niter", [0, 1, 7])
def test_press_adjoint_dot_products(require_gpu, case, niter):
    y = rand_fields(OUT, 100 + niter)
    g = press_b(case, y, niter)
    for s in range(3):
        x = rand_fields(IN, 200 + 10 * niter + s)
        check_dot(press64(case, x, niter), y, x, g, OUT, IN)


def test_press_adjoint_rejects_negative_count(require_gpu, case):
    y = rand_fields(OUT, 7)
    with pytest.raises(abi.LesError):
        press_b(case, y, -1)


VEL_IN, VEL_OUT = ["p", "u", "v", "w", "f", "g", "h"], ["u", "v", "w"]


def test_velnw_adjoint_dot_products(require_gpu, case):
    A, pr = case.arrays, case.params
    L = fp64.lib()
    i, d, p = C.c_int, C.c_double, C.c_void_p
    L.oracle_velnw.argtypes = [i, i, i, p, d, p, p, d, p, p, p, p, p, p, p]
    y = rand_fields(VEL_OUT, 31)
    b = {n: y[n].copy(order="F") for n in VEL_OUT}
    b.update({n: FL.alloc(n, IP, JP, KP) for n in ("p", "f", "g", "h")})
    Fp = FL.ptr
    abi.check(abi.lib().les_velnw_b_(I(KP), I(JP), I(IP), Fp(b["p"]), Fv(pr.ro), Fp(A["dxs"]), Fp(b["u"]),
                                     Fv(pr.dt), Fp(b["f"]), Fp(A["dys"]), Fp(b["v"]), Fp(b["g"]), Fp(A["dzs"]),
                                     Fp(b["w"]), Fp(b["h"])))
    co = {n: f64(A[n]) for n in ("dxs", "dys", "dzs")}
    for s in range(3):
        x = rand_fields(VEL_IN, 40 + s)
        a = {n: f64(x[n]) for n in VEL_IN}
        P = lambda n: a[n].ctypes.data
        L.oracle_velnw(KP, JP, IP, P("p"), float(np.float32(pr.ro)), co["dxs"].ctypes.data, P("u"),
                       float(np.float32(pr.dt)), P("f"), co["dys"].ctypes.data, P("v"), P("g"),
                       co["dzs"].ctypes.data, P("w"), P("h"))
        check_dot(a, y, x, b, VEL_OUT, VEL_IN)


FB_MASK = ["bmask1", "cmask1", "dmask1"]
FB_IN = ["usum", "u", "vsum", "v", "wsum", "w", "fx", "fy", "fz", "f", "g", "h"]
FB_OUT = ["usum", "vsum", "wsum", "fx", "fy", "fz", "f", "g", "h"]


def test_feedbf_adjoint_dot_products(require_gpu, case):
    A, pr = case.arrays, case.params
    L = fp64.lib()
    i, d, p = C.c_int, C.c_double, C.c_void_p
    L.oracle_feedbf.argtypes = [i, i, i] + [p] * 9 + [d, d, d] + [p] * 6
    alloc = {"fx": "f", "fy": "f", "fz": "f"}  # fx..fz have f's bounds (0:ip, 0:jp, 0:kp)
    y = {}
    rng = np.random.default_rng(51)
    for n in FB_OUT:
        a = FL.alloc(alloc.get(n, n), IP, JP, KP)
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
        y[n] = a
    b = {n: y[n].copy(order="F") for n in FB_OUT}
    b.update({n: FL.alloc(n, IP, JP, KP) for n in ("u", "v", "w")})
    Fp = FL.ptr
    abi.check(abi.lib().les_feedbf_b_(
        I(KP), I(JP), I(IP), Fp(b["usum"]), Fp(b["u"]), Fp(A["bmask1"]), Fp(b["vsum"]), Fp(b["v"]),
        Fp(A["cmask1"]), Fp(b["wsum"]), Fp(b["w"]), Fp(A["dmask1"]), Fv(pr.alpha), Fv(pr.dt), Fv(pr.beta),
        Fp(b["fx"]), Fp(b["fy"]), Fp(b["fz"]), Fp(b["f"]), Fp(b["g"]), Fp(b["h"])))
    m = {n: f64(A[n]) for n in FB_MASK}
    for s in range(3):
        rng = np.random.default_rng(60 + s)
        x = {}
        for n in FB_IN:
            a = FL.alloc(alloc.get(n, n), IP, JP, KP)
            a[...] = rng.standard_normal(a.shape).astype(np.float32)
            x[n] = a
        a = {n: f64(x[n]) for n in FB_IN}
        P = lambda n: a[n].ctypes.data
        L.oracle_feedbf(KP, JP, IP, P("usum"), P("u"), m["bmask1"].ctypes.data, P("vsum"), P("v"),
                        m["cmask1"].ctypes.data, P("wsum"), P("w"), m["dmask1"].ctypes.data,
                        float(np.float32(pr.alpha)), float(np.float32(pr.dt)), float(np.float32(pr.beta)),
                        P("fx"), P("fy"), P("fz"), P("f"), P("g"), P("h"))
        check_dot(a, y, x, b, FB_OUT, FB_IN)


ADAM = ["fold", "gold", "hold", "f", "g", "h"]


def test_adam_adjoint_dot_products(require_gpu, case):
    L = fp64.lib()
    i, p = C.c_int, C.c_void_p
    L.oracle_adam.argtypes = [i, i, p, i, i, i, p, p, p, p, p]
    y = rand_fields(ADAM, 71)
    b = {n: y[n].copy(order="F") for n in ADAM}
    Fp = FL.ptr
    abi.check(abi.lib().les_adam_b_(I(3), I(10), Fp(b["fold"]), I(IP), I(JP), I(KP), Fp(b["gold"]),
                                    Fp(b["hold"]), Fp(b["f"]), Fp(b["g"]), Fp(b["h"])))
    for s in range(3):
        x = rand_fields(ADAM, 80 + s)
        a = {n: f64(x[n]) for n in ADAM}
        P = lambda n: a[n].ctypes.data
        L.oracle_adam(3, 10, P("fold"), IP, JP, KP, P("gold"), P("hold"), P("f"), P("g"), P("h"))
        check_dot(a, y, x, b, ADAM, ADAM)


DIU = [f"diu{n}" for n in range(1, 10)]
LES_OUT = ["sm", "f", "g", "h"]


def les64(case, x):
    """The FP64 oracle's les on float64 copies; returns sm, f, g, h."""
    L = fp64.lib()
    i, p = C.c_int, C.c_void_p
    L.oracle_les.argtypes = [i, p, p, p, p, i, i] + [p] * 13
    a = {n: np.asfortranarray(np.asarray(x[n], dtype=np.float64)) for n in DIU + LES_OUT}
    co = {n: f64(case.arrays[n]) for n in ("dx1", "dy1", "dzn")}
    delx1 = np.zeros(KP)
    L.oracle_les(KP, delx1.ctypes.data, co["dx1"].ctypes.data, co["dy1"].ctypes.data, co["dzn"].ctypes.data, JP,
                 IP, *[a[n].ctypes.data for n in DIU + LES_OUT])
    return {n: a[n] for n in LES_OUT}


def test_les_adjoint_against_fp64_differences(require_gpu, case):
    """les is nonlinear: <J d, y> by central differences of the FP64 oracle
    (step 1e-5, error ~1e-10) against <d, J^T y> from les_les_b_ at the
    same state; random diu keep every strain invariant positive."""
    A = case.arrays
    x0 = rand_fields(DIU + LES_OUT, 300)
    y = rand_fields(LES_OUT, 301)
    b = {n: FL.alloc(n, IP, JP, KP) for n in DIU}
    b.update({n: y[n].copy(order="F") for n in LES_OUT})
    Fp = FL.ptr
    abi.check(abi.lib().les_les_b_(I(KP), Fp(A["dx1"]), Fp(A["dy1"]), Fp(A["dzn"]), I(JP), I(IP),
                                   *[Fp(x0[n]) for n in DIU], *[Fp(b[n]) for n in DIU],
                                   *[Fp(b[n]) for n in LES_OUT]))
    h = 1e-5
    for s in range(2):
        d = rand_fields(DIU + LES_OUT, 310 + s)
        xp = {n: x0[n].astype(np.float64) + h * d[n] for n in DIU + LES_OUT}
        xm = {n: x0[n].astype(np.float64) - h * d[n] for n in DIU + LES_OUT}
        fp, fm = les64(case, xp), les64(case, xm)
        jd = {n: (fp[n] - fm[n]) / (2 * h) for n in LES_OUT}
        check_dot(jd, y, d, b, LES_OUT, DIU + LES_OUT)
