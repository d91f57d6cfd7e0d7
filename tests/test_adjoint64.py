"""The FP64 reference adjoints of oracle/adjoint64.py against central
differences of the FP64 oracle (no GPU).

velfg (vel2.f95:48-188 + velFG.f95:56-105) is quadratic in (u, v, w): for
random (u, v, w), directions d and output seeds y on f, g, h and diu1..9,
<(F(x + h d) - F(x - h d)) / 2h, y> must equal <d, J^T y> from velfg_b to the
differences' accuracy (exact for a quadratic map up to FP64 rounding)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import adjoint64, fp64
from les_halo_b200 import fields as FL, synthetic_case

IP, JP, KP = 12, 10, 7
WORK = [f"{a}{n}" for n in range(1, 10) for a in ("nou", "diu", "cov")] + ["dfu1", "dfv1", "dfw1"]


def rnd(name, seed):
    a = FL.alloc(name, IP, JP, KP)
    a[...] = np.random.default_rng(seed).standard_normal(a.shape)
    return np.asfortranarray(a.astype(np.float64))


def velfg64(case, u, v, w):
    """FP64 oracle velfg from zeroed work arrays; returns f, g, h, diu1..9."""
    L = fp64.lib()
    i, d, p = C.c_int, C.c_double, C.c_void_p
    L.oracle_velfg.argtypes = [i, i, i] + [p] * 10 + [d] + [p] * 30
    a = {n: np.asfortranarray(np.zeros(FL.alloc(n, IP, JP, KP).shape)) for n in WORK + ["f", "g", "h"]}
    a.update({"u": np.asfortranarray(u), "v": np.asfortranarray(v), "w": np.asfortranarray(w)})
    co = {n: np.asfortranarray(case.arrays[n].astype(np.float64)) for n in ("dx1", "dy1", "dzn", "dzs")}
    P = lambda n: (a[n] if n in a else co[n]).ctypes.data
    order = ["dx1", "cov1", "cov2", "cov3", "dfu1", "diu1", "diu2", "dy1", "diu3", "dzn"]
    order2 = ["f", "cov4", "cov5", "cov6", "dfv1", "diu4", "diu5", "diu6", "g", "cov7", "cov8", "cov9", "dfw1",
              "diu7", "diu8", "diu9", "dzs", "h", "nou1", "u", "nou5", "v", "nou9", "w", "nou2", "nou3", "nou4",
              "nou6", "nou7", "nou8"]
    L.oracle_velfg(KP, JP, IP, *[P(n) for n in order], float(np.float32(case.params.vn)), *[P(n) for n in order2])
    return a


def test_velfg_reference_adjoint_against_fp64_differences():
    case = synthetic_case(IP, JP, KP, seed=3, masks_and_poisson=oracle.masks_and_poisson)
    x = {n: rnd(n, s) for s, n in enumerate(("u", "v", "w"))}
    outs = ["f", "g", "h"] + [f"diu{n}" for n in range(1, 10)]
    y = {n: rnd(n, 20 + s) for s, n in enumerate(outs)}
    metrics = {n: case.arrays[n].astype(np.float64) for n in ("dx1", "dy1", "dzn", "dzs")}
    (ub, vb, wb), _ = adjoint64.velfg_b(IP, JP, KP, metrics, float(np.float32(case.params.vn)), x["u"], x["v"],
                                        x["w"], y["f"], y["g"], y["h"], {n: y[f"diu{n}"] for n in range(1, 10)})
    adj = {"u": ub, "v": vb, "w": wb}
    h = 1e-4
    for s in range(2):
        d = {n: rnd(n, 40 + 3 * s + t) for t, n in enumerate(("u", "v", "w"))}
        fp = velfg64(case, *[x[n] + h * d[n] for n in ("u", "v", "w")])
        fm = velfg64(case, *[x[n] - h * d[n] for n in ("u", "v", "w")])
        lhs = sum(float(np.sum((fp[n] - fm[n]) / (2 * h) * y[n])) for n in outs)
        terms = [d[n] * adj[n] for n in ("u", "v", "w")]
        rhs = sum(float(t.sum()) for t in terms)
        scale = sum(float(np.abs(t).sum()) for t in terms)
        assert abs(lhs - rhs) <= 1e-9 * scale, (s, lhs, rhs, scale)


def bondv1_ext64(case, n, wp, u, v, w):
    L = fp64.lib()
    i, d, p = C.c_int, C.c_double, C.c_void_p
    L.oracle_bondv1_ext_wind_profile.argtypes = [i, p, p, p, p, p, i, i, i, d, p, p]
    a = {"u": np.asfortranarray(u.copy()), "v": np.asfortranarray(v.copy()), "w": np.asfortranarray(w.copy())}
    co = {nm: np.asfortranarray(case.arrays[nm].astype(np.float64)) for nm in ("z2", "dzn", "dxs")}
    wpa = np.asfortranarray(wp)
    L.oracle_bondv1_ext_wind_profile(JP, a["u"].ctypes.data, co["z2"].ctypes.data, co["dzn"].ctypes.data,
                                     a["v"].ctypes.data, a["w"].ctypes.data, KP, n, IP,
                                     float(np.float32(case.params.dt)), co["dxs"].ctypes.data, wpa.ctypes.data)
    return a





@pytest.mark.parametrize("n", [1, 5])
def test_bondv1_reference_adjoint_against_fp64_differences(n):
    """bondv1 (external inflow profile) is piecewise linear; random states
    keep the max/min of u(im, ., .) unique and away from the kinks, so
    central differences of the FP64 oracle are exact to rounding."""
    case = synthetic_case(IP, JP, KP, seed=4, masks_and_poisson=oracle.masks_and_poisson)
    x = {nm: rnd(nm, 60 + s) for s, nm in enumerate(("u", "v", "w"))}
    x["wp"] = rnd("wind_profile", 63)
    y = {nm: rnd(nm, 70 + s) for s, nm in enumerate(("u", "v", "w"))}
    dt = float(np.float32(case.params.dt))
    ub, vb, wb, wpb = adjoint64.bondv1_ext_b(IP, JP, KP, case.arrays["dxs"].astype(np.float64), dt, n, x["wp"],
                                             x["u"], x["v"], x["w"], y["u"], y["v"], y["w"])
    adj = {"u": ub, "v": vb, "w": wb, "wp": wpb}
    h = 1e-6
    for s in range(2):
        d = {nm: rnd(nm if nm != "wp" else "wind_profile", 80 + 4 * s + t)
             for t, nm in enumerate(("u", "v", "w", "wp"))}
        fp = bondv1_ext64(case, n, x["wp"] + h * d["wp"], *[x[nm] + h * d[nm] for nm in ("u", "v", "w")])
        fm = bondv1_ext64(case, n, x["wp"] - h * d["wp"], *[x[nm] - h * d[nm] for nm in ("u", "v", "w")])
        lhs = sum(float(np.sum((fp[nm] - fm[nm]) / (2 * h) * y[nm])) for nm in ("u", "v", "w"))
        terms = [d[nm] * adj[nm] for nm in ("u", "v", "w", "wp")]
        rhs = sum(float(t.sum()) for t in terms)
        scale = sum(float(np.abs(t).sum()) for t in terms)
        assert abs(lhs - rhs) <= 1e-8 * scale, (n, s, lhs, rhs, scale)


@pytest.mark.parametrize("n", [1, 5])
def test_step_reference_adjoint_against_fp64_differences(n):
    """The whole step (velnw, bondv1 with the external inflow profile,
    velfg, feedbf, les, adam, press with 3 SOR iterations) composed from the
    reference adjoints, against central differences of the FP64 oracle's
    step over every state array and the inflow profile."""
    case = synthetic_case(IP, JP, KP, seed=6, masks_and_poisson=oracle.masks_and_poisson)
    names = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
             "cn3l", "cn3s", "cn4l", "cn4s"]
    co = {nm: case.arrays[nm] for nm in names}
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    step = adjoint64.Step64(IP, JP, KP, co, prm, 3)
    x = {nm: rnd(nm, 100 + s) for s, nm in enumerate(adjoint64.STATE)}
    wp = rnd("wind_profile", 99)
    y = {nm: rnd(nm, 200 + s) for s, nm in enumerate(adjoint64.STATE)}
    _, tape = step.forward(n, x, wp)
    adj, grads = step.adjoint(n, tape, wp, y)
    wpb = grads["wp"]
    h = 1e-6
    for s in range(2):
        d = {nm: rnd(nm, 300 + 20 * s + t) for t, nm in enumerate(adjoint64.STATE)}
        dwp = rnd("wind_profile", 399 + s)
        fp, _ = step.forward(n, {k: x[k] + h * d[k] for k in x}, wp + h * dwp)
        fm, _ = step.forward(n, {k: x[k] - h * d[k] for k in x}, wp - h * dwp)
        lhs = sum(float(np.sum((fp[k] - fm[k]) / (2 * h) * y[k])) for k in adjoint64.STATE)
        terms = [d[k] * adj[k] for k in adjoint64.STATE] + [dwp * wpb]
        rhs = sum(float(t.sum()) for t in terms)
        scale = sum(float(np.abs(t).sum()) for t in terms)
        assert abs(lhs - rhs) <= 1e-7 * scale, (n, s, lhs, rhs, scale, abs(lhs - rhs) / scale)


def test_tke_gradient_with_checkpoints_against_fp64_differences():
    """J = time- and box-mean resolved TKE over 4 steps (n = 1..4, SOR 3
    iterations, a checkpoint every 2 steps with recomputation): its gradient
    with respect to the inflow profile and the initial state against central
    differences of the FP64 oracle's steps."""
    case = synthetic_case(IP, JP, KP, seed=8, masks_and_poisson=oracle.masks_and_poisson)
    names = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
             "cn3l", "cn3s", "cn4l", "cn4s"]
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    step = adjoint64.Step64(IP, JP, KP, {nm: case.arrays[nm] for nm in names}, prm, 3)
    x = {nm: rnd(nm, 500 + s) for s, nm in enumerate(adjoint64.STATE)}
    wp = rnd("wind_profile", 499)
    box = ((3, 8), (2, 7), (1, 3))
    nt = 4
    J, grads, bar = adjoint64.tke_gradient(step, 1, nt, x, wp, box, ckpt=2)
    wpb = grads["wp"]

    def J_of(state, w):
        s, acc = state, 0.0
        for t in range(nt):
            s, _ = step.forward(1 + t, s, w)
            acc += adjoint64.tke(IP, JP, KP, s, box) / nt
        return acc

    assert abs(J - J_of(x, wp)) <= 1e-14 * abs(J)
    h = 1e-6
    dwp = rnd("wind_profile", 600)
    fd = (J_of(x, wp + h * dwp) - J_of(x, wp - h * dwp)) / (2 * h)
    ad = float(np.sum(dwp * wpb))
    assert abs(fd - ad) <= 1e-7 * float(np.sum(np.abs(dwp * wpb))), (fd, ad)
    d = {nm: rnd(nm, 700 + s) for s, nm in enumerate(adjoint64.STATE)}
    fd = (J_of({k: x[k] + h * d[k] for k in x}, wp) - J_of({k: x[k] - h * d[k] for k in x}, wp)) / (2 * h)
    terms = [d[k] * bar[k] for k in adjoint64.STATE]
    ad = sum(float(t.sum()) for t in terms)
    assert abs(fd - ad) <= 1e-7 * sum(float(np.abs(t).sum()) for t in terms), (fd, ad)


def test_tke_gradient_for_the_drag_scale():
    """The same objective with a per-column drag scale s(i, j) on feedbf's
    force (s = 1 reproduces the reference step bit for bit in FP64): its
    gradient with respect to s against central differences."""
    case = synthetic_case(IP, JP, KP, seed=9, masks_and_poisson=oracle.masks_and_poisson)
    names = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
             "cn3l", "cn3s", "cn4l", "cn4s"]
    co = {nm: case.arrays[nm] for nm in names}
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    x = {nm: rnd(nm, 800 + s) for s, nm in enumerate(adjoint64.STATE)}
    wp = rnd("wind_profile", 799)
    one = adjoint64.Step64(IP, JP, KP, co, prm, 3, drag=np.ones((IP, JP)))
    ref = adjoint64.Step64(IP, JP, KP, co, prm, 3)
    a1, _ = one.forward(2, x, wp)
    a0, _ = ref.forward(2, x, wp)
    assert all(np.array_equal(a1[k], a0[k]) for k in adjoint64.STATE)
    drag = 1.0 + 0.3 * np.random.default_rng(5).standard_normal((IP, JP))
    box, nt = ((3, 8), (2, 7), (1, 3)), 3
    step = adjoint64.Step64(IP, JP, KP, co, prm, 3, drag=drag)
    J, grads, _ = adjoint64.tke_gradient(step, 2, nt, x, wp, box, ckpt=2)

    def J_of(dr):
        st = adjoint64.Step64(IP, JP, KP, co, prm, 3, drag=dr)
        s, acc = x, 0.0
        for t in range(nt):
            s, _ = st.forward(2 + t, s, wp)
            acc += adjoint64.tke(IP, JP, KP, s, box) / nt
        return acc

    h = 1e-6
    dd = np.random.default_rng(6).standard_normal((IP, JP))
    fd = (J_of(drag + h * dd) - J_of(drag - h * dd)) / (2 * h)
    ad = float(np.sum(dd * grads["drag"]))
    assert abs(fd - ad) <= 1e-7 * float(np.sum(np.abs(dd * grads["drag"]))), (fd, ad)


def _ref_case(seed):
    case = synthetic_case(IP, JP, KP, seed=seed, masks_and_poisson=oracle.masks_and_poisson)
    names = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
             "cn3l", "cn3s", "cn4l", "cn4s"]
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    return {nm: case.arrays[nm].astype(np.float64) for nm in names}, prm


def _dot_check(lhs_out, y, d, adj, tol):
    lhs = sum(float(np.sum(lhs_out[k] * y[k])) for k in y)
    terms = [d[k] * adj[k] for k in d]
    rhs = sum(float(t.sum()) for t in terms)
    assert abs(lhs - rhs) <= tol * sum(float(np.abs(t).sum()) for t in terms), (lhs, rhs)


def test_press_reference_adjoint_dot_products():
    co, prm = _ref_case(12)
    step = adjoint64.Step64(IP, JP, KP, co, prm, 4)  # for its bound oracle_press_ex
    L = step.L
    outs, ins = ["rhs", "p", "f", "g", "h"], ["rhs", "u", "v", "w", "f", "g", "h", "p"]
    y = {k: rnd(k, 1000 + s) for s, k in enumerate(outs)}
    (rb, pb, fb, gb, hb), (ub, vb, wb) = adjoint64.press_b(IP, JP, KP, co, prm["dt"], prm["omega"], 4, y["rhs"],
                                                           y["p"], y["f"], y["g"], y["h"])
    adj = {"rhs": rb, "p": pb, "f": fb, "g": gb, "h": hb, "u": ub, "v": vb, "w": wb}
    x = {k: rnd(k, 1100 + s) for s, k in enumerate(ins)}
    a = {k: np.asfortranarray(x[k].copy()) for k in ins}
    c = {k: np.asfortranarray(co[k]) for k in co}
    P = lambda k: (a[k] if k in a else c[k]).ctypes.data
    L.oracle_press_ex(KP, JP, IP, P("rhs"), P("u"), P("dx1"), P("v"), P("dy1"), P("w"), P("dzn"), P("f"), P("g"),
                      P("h"), prm["dt"], P("cn1"), P("cn2l"), P("p"), P("cn2s"), P("cn3l"), P("cn3s"), P("cn4l"),
                      P("cn4s"), 4, -1.0, prm["omega"], None, None, None)
    _dot_check({k: a[k] for k in outs}, y, x, adj, 1e-12)


def test_les_reference_adjoint_against_fp64_differences():
    co, prm = _ref_case(13)
    step = adjoint64.Step64(IP, JP, KP, co, prm, 1)
    L = step.L
    diu = {n: rnd(f"diu{n}", 1200 + n) for n in range(1, 10)}
    outs = ["sm", "f", "g", "h"]
    y = {k: rnd(k, 1300 + s) for s, k in enumerate(outs)}
    smb, diub = adjoint64.les_b(IP, JP, KP, co, diu, y["sm"], y["f"], y["g"], y["h"])
    adj = {"sm": smb, "f": y["f"], "g": y["g"], "h": y["h"], **{f"diu{n}": diub[n] for n in range(1, 10)}}
    base = {k: rnd(k, 1400 + s) for s, k in enumerate(outs)}
    d = {k: rnd(k, 1500 + s) for s, k in enumerate(list(adj))}

    def run(sign, h=1e-6):
        a = {k: np.asfortranarray(base[k] + sign * h * d[k]) for k in outs}
        a.update({f"diu{n}": np.asfortranarray(diu[n] + sign * h * d[f"diu{n}"]) for n in range(1, 10)})
        c = {k: np.asfortranarray(co[k]) for k in ("dx1", "dy1", "dzn")}
        dl = np.zeros(KP)
        L.oracle_les(KP, dl.ctypes.data, c["dx1"].ctypes.data, c["dy1"].ctypes.data, c["dzn"].ctypes.data, JP, IP,
                     *[a[f"diu{n}"].ctypes.data for n in range(1, 10)], *[a[k].ctypes.data for k in outs])
        return a

    fp, fm = run(1.0), run(-1.0)
    _dot_check({k: (fp[k] - fm[k]) / 2e-6 for k in outs}, y, d, adj, 1e-8)
