"""FP64 reference adjoints (reverse mode) of the time step's routines and of
the whole step, in NumPy.

TEST INFRASTRUCTURE ONLY, like the rest of oracle/: the reference gradient
that the CUDA adjoint entries are checked against, itself checked against
central differences of the FP64 oracle (oracle/fp64.py) in
tests/test_adjoint64.py.

bondv1_ext_b: bondv1_ext_wind_profile.f95:27-127 (inflow from the external
profile, n == 1 broadcast, outflow with uout, periodic, top and ground).

velnw_b, feedbf_b, adam_b, press_b, les_b restate in FP64 the transposes the
CUDA entries les_velnw_b_ .. les_les_b_ compute, and Step64 composes all of
them into the adjoint of one whole time step (the sequence of
oracle_run_steps, main_ocl.f95:264-299, with the external inflow profile
and a fixed SOR iteration count): the FP64 reference gradient of a step.

velfg_b: vel2.f95:48-188 + velFG.f95:56-105, the face quantities of (u, v,
w) and the advection/diffusion terms f, g, h.  The map is quadratic (cov =
nou * diu); its adjoint is taken at the given (u, v, w).  Outputs whose
adjoints are taken: f, g, h and diu1..9 (les reads diu).  nou*, cov* and
dfu1/dfv1/dfw1 are work arrays the next call recomputes; their seeds are
not inputs here, and the adjoint with respect to the previous contents of
any array the routine overwrites is not returned.
"""
from __future__ import annotations

import numpy as np

from les_halo_b200 import fields as FL


class FA:
    """A float64 array with Fortran lower bounds: a[i, j, k] takes Fortran
    indices or inclusive (lo, hi) ranges."""

    def __init__(self, name, ip, jp, kp, arr=None):
        self.lo = [FL._ev(b.split(":")[0], ip, jp, kp) for b in FL._BOUNDS[name]]
        self.arr = np.zeros(FL.alloc(name, ip, jp, kp).shape) if arr is None else arr

    def _sl(self, idx):
        return tuple(slice(a[0] - l, a[1] - l + 1) if isinstance(a, tuple) else a - l
                     for a, l in zip(idx, self.lo))

    def __getitem__(self, idx):
        return self.arr[self._sl(idx)]

    def __setitem__(self, idx, v):
        self.arr[self._sl(idx)] = v


def _m1(a, lo, rng, axis):
    """1-D metric a (Fortran lower bound lo) over the inclusive range rng,
    shaped to broadcast along `axis` of a 3-D block."""
    v = np.asarray(a, dtype=np.float64)[rng[0] - lo:rng[1] - lo + 1]
    shape = [1, 1, 1]
    shape[axis] = v.size
    return v.reshape(shape)


def velfg_b(ip, jp, kp, metrics, vn, u, v, w, fb, gb, hb, diub):
    """Adjoint of velfg at (u, v, w).  metrics: dx1, dy1, dzn, dzs (Fortran
    layout); u, v, w, fb, gb, hb and diub[n] (n = 1..9) float arrays with the
    routines' Fortran bounds.  Returns (ub, vb, wb) (the adjoints of u, v, w)
    and the diu adjoints after the boundary copies (for inspection)."""
    im, jm, km = ip, jp, kp
    U, V, W = (FA(n, ip, jp, kp, np.asarray(a, dtype=np.float64)) for n, a in (("u", u), ("v", v), ("w", w)))
    ub, vb, wb = FA("u", ip, jp, kp), FA("v", ip, jp, kp), FA("w", ip, jp, kp)
    X = lambda r: _m1(metrics["dx1"], -1, r, 0)
    Y = lambda r: _m1(metrics["dy1"], 0, r, 1)
    Zn = lambda r: _m1(metrics["dzn"], -1, r, 2)
    Zs = lambda r: _m1(metrics["dzs"], -1, r, 2)
    I, J, K = (1, im), (1, jm), (1, km)
    sh = lambda r, d: (r[0] + d, r[1] + d)
    names = {n: (f"nou{n}", f"diu{n}", f"cov{n}") for n in range(1, 10)}
    nb = {n: FA(names[n][0], ip, jp, kp) for n in range(1, 10)}
    db = {n: FA(names[n][1], ip, jp, kp, np.asarray(diub[n], dtype=np.float64).copy()) for n in range(1, 10)}
    cb = {n: FA(names[n][2], ip, jp, kp) for n in range(1, 10)}

    # --- velFG.f95:56-105 transposed (f, g, h overwritten on their ranges)
    Fb, Gb, Hb = (FA(n, ip, jp, kp, np.asarray(a, dtype=np.float64)) for n, a in (("f", fb), ("g", gb), ("h", hb)))
    s = -Fb[I, J, K]  # covc's adjoint
    d = vn * Fb[I, J, K]  # dfu1's
    sx = X(sh(I, 0)) + X(sh(I, 1))
    cb[1][I, J, K] += s * X(sh(I, 1)) / sx
    cb[1][sh(I, 1), J, K] += s * X(I) / sx
    cb[2][I, J, K] += s / 2.0
    cb[2][I, sh(J, 1), K] += s / 2.0
    cb[3][I, J, K] += s / 2.0
    cb[3][I, J, sh(K, 1)] += s / 2.0
    db[1][I, J, K] -= 2.0 * d / sx
    db[1][sh(I, 1), J, K] += 2.0 * d / sx
    db[2][I, J, K] -= d / Y(J)
    db[2][I, sh(J, 1), K] += d / Y(J)
    db[3][I, J, K] -= d / Zn(K)
    db[3][I, J, sh(K, 1)] += d / Zn(K)

    s = -Gb[I, J, K]
    d = vn * Gb[I, J, K]
    sy = Y(J) + Y(sh(J, 1))
    cb[4][I, J, K] += s / 2.0
    cb[4][sh(I, 1), J, K] += s / 2.0
    cb[5][I, J, K] += s * Y(sh(J, 1)) / sy
    cb[5][I, sh(J, 1), K] += s * Y(J) / sy
    cb[6][I, J, K] += s / 2.0
    cb[6][I, J, sh(K, 1)] += s / 2.0
    db[4][I, J, K] -= d / X(I)
    db[4][sh(I, 1), J, K] += d / X(I)
    db[5][I, J, K] -= 2.0 * d / sy
    db[5][I, sh(J, 1), K] += 2.0 * d / sy
    db[6][I, J, K] -= d / Zn(K)
    db[6][I, J, sh(K, 1)] += d / Zn(K)

    K1 = (1, km - 1)
    s = -Hb[I, J, K1]
    d = vn * Hb[I, J, K1]
    sz = Zn(K1) + Zn(sh(K1, 1))
    cb[7][I, J, K1] += s / 2.0
    cb[7][sh(I, 1), J, K1] += s / 2.0
    cb[8][I, J, K1] += s / 2.0
    cb[8][I, sh(J, 1), K1] += s / 2.0
    cb[9][I, J, K1] += s * Zn(sh(K1, 1)) / sz
    cb[9][I, J, sh(K1, 1)] += s * Zn(K1) / sz
    db[7][I, J, K1] -= d / X(I)
    db[7][sh(I, 1), J, K1] += d / X(I)
    db[8][I, J, K1] -= d / Y(J)
    db[8][I, sh(J, 1), K1] += d / Y(J)
    db[9][I, J, K1] -= d / Zs(K1)
    db[9][I, J, sh(K1, 1)] += d / Zs(K1)

    # --- vel2.f95:125-188 boundary copies transposed, last first; dst = src
    # becomes src_b += dst_b, dst_b = 0 (statement by statement)
    def mv(arr, dst, src):
        arr[src] += arr[dst]
        arr[dst] = 0.0

    def mv_each(arrs, loops):
        for a in arrs:
            for dst, src in loops:
                mv(a, dst, src)

    Kp1, Ip1, Jp1 = (1, km + 1), (1, im + 1), (1, jm + 1)
    mv_each([db[6], db[4]], [((Ip1, 0, Kp1), (Ip1, jm, Kp1))])
    mv_each([db[3], db[2]], [((im + 1, Jp1, Kp1), (im, Jp1, Kp1))])
    for n, kr in ((8, K1), (5, K), (2, K)):  # j copies: x(.,0) = x(.,jm); x(.,jm+1) = x(.,1)
        for a in (cb[n], db[n], nb[n]):
            mv(a, (I, jm + 1, kr), (I, 1, kr))
            mv(a, (I, 0, kr), (I, jm, kr))
        if n == 8:
            for a in (cb[7], db[7], nb[7]):
                mv(a, (im + 1, J, K1), (im, J, K1))
        if n == 5:
            for a in (cb[4], db[4], nb[4]):
                mv(a, (im + 1, J, K), (im, J, K))
    for a in (cb[1], db[1], nb[1]):
        mv(a, (im + 1, J, K), (im, J, K))

    # --- vel2.f95:48-123 transposed: cov = nou * diu at the forward values,
    # then nou and diu back to u, v, w
    def face(n, ir, jr, kr, nou, diu):
        c = cb[n][ir, jr, kr]
        return nb[n][ir, jr, kr] + c * diu, db[n][ir, jr, kr] + c * nou

    # 1, 5, 9: centred differences along x, y, z
    nou = (U[sh(I, -1), J, K] + U[I, J, K]) / 2.0
    diu = (-U[sh(I, -1), J, K] + U[I, J, K]) / X(I)
    a, b = face(1, I, J, K, nou, diu)
    ub[sh(I, -1), J, K] += a / 2.0 - b / X(I)
    ub[I, J, K] += a / 2.0 + b / X(I)
    nou = (V[I, sh(J, -1), K] + V[I, J, K]) / 2.0
    diu = (-V[I, sh(J, -1), K] + V[I, J, K]) / Y(J)
    a, b = face(5, I, J, K, nou, diu)
    vb[I, sh(J, -1), K] += a / 2.0 - b / Y(J)
    vb[I, J, K] += a / 2.0 + b / Y(J)
    nou = (W[I, J, sh(K, -1)] + W[I, J, K]) / 2.0
    diu = (-W[I, J, sh(K, -1)] + W[I, J, K]) / Zn(K)
    a, b = face(9, I, J, K, nou, diu)
    wb[I, J, sh(K, -1)] += a / 2.0 - b / Zn(K)
    wb[I, J, K] += a / 2.0 + b / Zn(K)
    # 2: nou from v (x pair), diu from u along y
    sx = X(I) + X(sh(I, 1))
    sy = Y(sh(J, -1)) + Y(J)
    nou = (X(sh(I, 1)) * V[I, sh(J, -1), K] + X(I) * V[sh(I, 1), sh(J, -1), K]) / sx
    diu = 2.0 * (-U[I, sh(J, -1), K] + U[I, J, K]) / sy
    a, b = face(2, I, J, K, nou, diu)
    vb[I, sh(J, -1), K] += a * X(sh(I, 1)) / sx
    vb[sh(I, 1), sh(J, -1), K] += a * X(I) / sx
    ub[I, sh(J, -1), K] -= 2.0 * b / sy
    ub[I, J, K] += 2.0 * b / sy
    # 3: nou from w (x pair, plane k-1), diu from u along z (k = 1..km+1)
    nou = (X(sh(I, 1)) * W[I, J, sh(Kp1, -1)] + X(I) * W[sh(I, 1), J, sh(Kp1, -1)]) / sx
    diu = (-U[I, J, sh(Kp1, -1)] + U[I, J, Kp1]) / Zs(sh(Kp1, -1))
    a, b = face(3, I, J, Kp1, nou, diu)
    wb[I, J, sh(Kp1, -1)] += a * X(sh(I, 1)) / sx
    wb[sh(I, 1), J, sh(Kp1, -1)] += a * X(I) / sx
    ub[I, J, sh(Kp1, -1)] -= b / Zs(sh(Kp1, -1))
    ub[I, J, Kp1] += b / Zs(sh(Kp1, -1))
    # 4: nou from u (column i-1, y pair), diu from v along x
    sy1 = Y(J) + Y(sh(J, 1))
    sxm = X(sh(I, -1)) + X(I)
    nou = (Y(sh(J, 1)) * U[sh(I, -1), J, K] + Y(J) * U[sh(I, -1), sh(J, 1), K]) / sy1
    diu = 2.0 * (-V[sh(I, -1), J, K] + V[I, J, K]) / sxm
    a, b = face(4, I, J, K, nou, diu)  # u0 = 0 (vel2.f95:46)
    ub[sh(I, -1), J, K] += a * Y(sh(J, 1)) / sy1
    ub[sh(I, -1), sh(J, 1), K] += a * Y(J) / sy1
    vb[sh(I, -1), J, K] -= 2.0 * b / sxm
    vb[I, J, K] += 2.0 * b / sxm
    # 6: nou from w (y pair, plane k-1), diu from v along z (k = 1..km+1)
    nou = (Y(sh(J, 1)) * W[I, J, sh(Kp1, -1)] + Y(J) * W[I, sh(J, 1), sh(Kp1, -1)]) / sy1
    diu = (-V[I, J, sh(Kp1, -1)] + V[I, J, Kp1]) / Zs(sh(Kp1, -1))
    a, b = face(6, I, J, Kp1, nou, diu)
    wb[I, J, sh(Kp1, -1)] += a * Y(sh(J, 1)) / sy1
    wb[I, sh(J, 1), sh(Kp1, -1)] += a * Y(J) / sy1
    vb[I, J, sh(Kp1, -1)] -= b / Zs(sh(Kp1, -1))
    vb[I, J, Kp1] += b / Zs(sh(Kp1, -1))
    # 7: nou from u (column i-1, z pair), diu from w along x (k = 1..km-1)
    sz = Zn(K1) + Zn(sh(K1, 1))
    nou = (Zn(sh(K1, 1)) * U[sh(I, -1), J, K1] + Zn(K1) * U[sh(I, -1), J, sh(K1, 1)]) / sz
    diu = 2.0 * (-W[sh(I, -1), J, K1] + W[I, J, K1]) / sxm
    a, b = face(7, I, J, K1, nou, diu)
    ub[sh(I, -1), J, K1] += a * Zn(sh(K1, 1)) / sz
    ub[sh(I, -1), J, sh(K1, 1)] += a * Zn(K1) / sz
    wb[sh(I, -1), J, K1] -= 2.0 * b / sxm
    wb[I, J, K1] += 2.0 * b / sxm
    # 8: nou from v (row j-1, z pair), diu from w along y (k = 1..km-1)
    nou = (Zn(sh(K1, 1)) * V[I, sh(J, -1), K1] + Zn(K1) * V[I, sh(J, -1), sh(K1, 1)]) / sz
    diu = 2.0 * (-W[I, sh(J, -1), K1] + W[I, J, K1]) / sy
    a, b = face(8, I, J, K1, nou, diu)
    vb[I, sh(J, -1), K1] += a * Zn(sh(K1, 1)) / sz
    vb[I, sh(J, -1), sh(K1, 1)] += a * Zn(K1) / sz
    wb[I, sh(J, -1), K1] -= 2.0 * b / sy
    wb[I, J, K1] += 2.0 * b / sy
    return (ub.arr, vb.arr, wb.arr), {n: db[n].arr for n in range(1, 10)}


def bondv1_ext_b(ip, jp, kp, dxs, dt, n, wp, u, v, w, ub, vb, wb):
    """Adjoint of bondv1_ext_wind_profile.f95:27-127 at the state (u, v, w)
    and wind profile wp(j, k) it is called with.  ub, vb, wb: adjoints of its
    outputs u, v, w.
    Returns (ub, vb, wb, wpb): the adjoints of its inputs u, v, w and of the
    wind profile wp(j, k).  Piecewise linear: uout = (max(0, u(im,.,.)) +
    min(0, u(im,.,.)))/2 passes its derivative to the first maximal (and
    minimal) element in the reference's loop order (k outer, j inner), as
    amax1/amin1 pick it; a tie or a zero extreme has no derivative there."""
    im, jm, km = ip, jp, kp
    U, V, W = (FA(nm, ip, jp, kp, np.asarray(a, dtype=np.float64).copy()) for nm, a in (("u", u), ("v", v), ("w", w)))
    Ub, Vb, Wb = (FA(nm, ip, jp, kp, np.asarray(a, dtype=np.float64).copy()) for nm, a in (("u", ub), ("v", vb), ("w", wb)))
    J, K = (1, jm), (1, km)
    ds = float(np.asarray(dxs, dtype=np.float64)[im])  # dxs(0:ip)
    # forward up to the tail: inflow (bondv1_ext_wind_profile.f95:27-34) is
    # overwritten data; the n == 1 broadcast (bondv1.f95:47-59) copies i = 1
    U[(0, 1), J, K] = np.asarray(wp, dtype=np.float64)[np.newaxis, :, :]
    V[(0, 1), J, K] = 0.0
    W[(0, 1), J, K] = 0.0
    if n == 1:
        for A in (U, V, W):
            A[(2, im), J, K] = A[1, J, K][np.newaxis, :, :]
    # primal values the tail reads (before its updates)
    u_im = U[im, J, K].copy()
    du = U[im, J, K] - U[im - 1, J, K]
    dvv = V[im + 1, J, K] - V[im, J, K]
    dww = W[im + 1, J, K] - W[im, J, K]
    aaa = max(0.0, float(u_im.max()))
    bbb = min(0.0, float(u_im.min()))
    uout = (aaa + bbb) / 2.0
    c = dt * uout / ds

    # w(., ., 0) = w(., ., km) = 0 for i = -1..im+1, j = -1..jm+1; i = -1 is
    # w(ip+1, j-1, .) in the column-major layout (j = -1: w(ip+1, jp+1, k-1))
    Wb[(0, im + 1), (-1, jm + 1), 0] = 0.0
    Wb[(0, im + 1), (-1, jm + 1), km] = 0.0
    Wb[ip + 1, (-1, jm), 0] = 0.0
    Wb[ip + 1, (-1, jm), km] = 0.0
    Wb[ip + 1, jp + 1, -1] = 0.0
    Wb[ip + 1, jp + 1, km - 1] = 0.0
    # top and ground, v then u: x(.,.,0) = -x(.,.,1); x(.,.,km+1) = x(.,.,km)
    for A in (Vb, Ub):
        A[(0, im + 1), (0, jm + 1), km] += A[(0, im + 1), (0, jm + 1), km + 1]
        A[(0, im + 1), (0, jm + 1), km + 1] = 0.0
        A[(0, im + 1), (0, jm + 1), 1] -= A[(0, im + 1), (0, jm + 1), 0]
        A[(0, im + 1), (0, jm + 1), 0] = 0.0
    # periodic j, w (k = 0..km) then v, u (k = 0..km+1)
    for A, kr in ((Wb, (0, km)), (Vb, (0, km + 1)), (Ub, (0, km + 1))):
        A[(0, im + 1), 1, kr] += A[(0, im + 1), jm + 1, kr]
        A[(0, im + 1), jm + 1, kr] = 0.0
        A[(0, im + 1), jm, kr] += A[(0, im + 1), 0, kr]
        A[(0, im + 1), 0, kr] = 0.0
    # outflow, w then v then u: x(e) = x(e) - (dt*uout)*(x(e) - x(e-1))/dxs(im)
    uoutb = 0.0
    for A, e, dx in ((Wb, im + 1, dww), (Vb, im + 1, dvv), (Ub, im, du)):
        ob = A[e, J, K].copy()
        uoutb += float(np.sum(-dt / ds * dx * ob))
        A[e - 1, J, K] += c * ob
        A[e, J, K] = (1.0 - c) * ob
    # uout = (aaa + bbb)/2 over u(im, 1..jm, 1..km), first extreme in k-major order
    order = u_im.T  # [k, j]
    if aaa > 0.0:
        kk, jj = np.unravel_index(int(np.argmax(order)), order.shape)
        Ub[im, 1 + jj, 1 + kk] += uoutb / 2.0
    if bbb < 0.0:
        kk, jj = np.unravel_index(int(np.argmin(order)), order.shape)
        Ub[im, 1 + jj, 1 + kk] += uoutb / 2.0
    # n == 1 broadcast: x(i, j, k) = x(1, j, k), i = 2..im
    if n == 1:
        for A in (Ub, Vb, Wb):
            A[1, J, K] += A[(2, im), J, K].sum(axis=0)
            A[(2, im), J, K] = 0.0
    # inflow: u(0:1, j, k) = wp(j, k); v = w = 0 there
    wpb = Ub[0, J, K] + Ub[1, J, K]
    for A in (Ub, Vb, Wb):
        A[(0, 1), J, K] = 0.0
    return Ub.arr, Vb.arr, Wb.arr, wpb


# ---- routines whose CUDA adjoint exists (les_adjoint.cuh), restated in FP64
# for the step-level reference below.  Each takes and returns full arrays
# with the routine's Fortran bounds; elements the routine never touches keep
# their adjoint.

def velnw_b(ip, jp, kp, dxs, dys, dzs, ro, dt, ub, vb, wb):
    """velnw.f95:27-59: u, v (all k), w (k <= km-1) += dt*(f - (p(+1) - p)/ro/ds).
    Returns the adjoint contributions (pb, fb, gb, hb); u, v, w keep theirs."""
    im, jm, km = ip, jp, kp
    Ub, Vb, Wb = (FA(n, ip, jp, kp, np.asarray(a, dtype=np.float64)) for n, a in (("u", ub), ("v", vb), ("w", wb)))
    Pb, Fb, Gb, Hb = FA("p", ip, jp, kp), FA("f", ip, jp, kp), FA("g", ip, jp, kp), FA("h", ip, jp, kp)
    I, J, K, K1 = (1, im), (1, jm), (1, km), (1, km - 1)
    sh = lambda r, d: (r[0] + d, r[1] + d)
    XS = _m1(dxs, 0, I, 0)
    YS = _m1(dys, 0, J, 1)
    ZS = _m1(dzs, -1, K1, 2)
    a = dt * Ub[I, J, K] / ro / XS
    Pb[sh(I, 1), J, K] -= a
    Pb[I, J, K] += a
    Fb[I, J, K] += dt * Ub[I, J, K]
    a = dt * Vb[I, J, K] / ro / YS
    Pb[I, sh(J, 1), K] -= a
    Pb[I, J, K] += a
    Gb[I, J, K] += dt * Vb[I, J, K]
    a = dt * Wb[I, J, K1] / ro / ZS
    Pb[I, J, sh(K1, 1)] -= a
    Pb[I, J, K1] += a
    Hb[I, J, K1] += dt * Wb[I, J, K1]
    return Pb.arr, Fb.arr, Gb.arr, Hb.arr


def feedbf_b(ip, jp, kp, masks, alpha, dt, beta, usumb, vsumb, wsumb, fb, gb, hb):
    """feedbf.f95:38-67 on the interior: sum' = (sum + v) m; fx = (alpha sum')
    dt + (beta v) m; f' = f + fx (fx a work array).  Returns the new
    (usumb, vsumb, wsumb) and the contributions (ub, vb, wb); f, g, h keep
    their adjoints."""
    I, J, K = (1, ip), (1, jp), (1, kp)
    out_s, out_v = [], []
    for sname, vname, mname, sb, xb in (("usum", "u", "bmask1", usumb, fb), ("vsum", "v", "cmask1", vsumb, gb),
                                        ("wsum", "w", "dmask1", wsumb, hb)):
        S = FA(sname, ip, jp, kp, np.asarray(sb, dtype=np.float64).copy())
        Vb = FA(vname, ip, jp, kp)
        M = FA(mname, ip, jp, kp, np.asarray(masks[mname], dtype=np.float64))
        X = FA("f", ip, jp, kp, np.asarray(xb, dtype=np.float64))
        m = M[I, J, K]
        t = X[I, J, K]
        s = S[I, J, K] + (alpha * dt) * t
        Vb[I, J, K] += (beta * m) * t + m * s
        S[I, J, K] = m * s
        out_s.append(S.arr)
        out_v.append(Vb.arr)
    return tuple(out_s), tuple(out_v)


def adam_b(ip, jp, kp, fb, gb, hb, foldb, goldb, holdb):
    """adam.f95:32-46: f' = 1.5 f - 0.5 fold, fold' = f on the interior."""
    I, J, K = (1, ip), (1, jp), (1, kp)
    res = []
    for nm, xb, ob in (("f", fb, foldb), ("g", gb, goldb), ("h", hb, holdb)):
        X = FA("f", ip, jp, kp, np.asarray(xb, dtype=np.float64).copy())
        O = FA("fold", ip, jp, kp, np.asarray(ob, dtype=np.float64).copy())
        x, o = X[I, J, K].copy(), O[I, J, K].copy()
        X[I, J, K] = 1.5 * x + o
        O[I, J, K] = -0.5 * x
        res.append((X.arr, O.arr))
    return res


def press_b(ip, jp, kp, co, dt, omega, niter, rhsb, pb, fb, gb, hb):
    """press.f95:49-146 with niter SOR iterations (the map is linear).  co:
    dx1, dy1, dzn, cn1, cn2l..cn4s (Fortran layout).  Takes the adjoints of
    the outputs rhs, p, f, g, h; returns those of the inputs (rhsb, pb, fb,
    gb, hb) and the contributions (ub, vb, wb)."""
    im, jm, km = ip, jp, kp
    R = FA("rhs", ip, jp, kp, np.asarray(rhsb, dtype=np.float64).copy())
    P = FA("p", ip, jp, kp, np.asarray(pb, dtype=np.float64).copy())
    Fb, Gb, Hb = (FA("f", ip, jp, kp, np.asarray(a, dtype=np.float64).copy()) for a in (fb, gb, hb))
    Ub, Vb, Wb = FA("u", ip, jp, kp), FA("v", ip, jp, kp), FA("w", ip, jp, kp)
    d = {n: np.asarray(co[n], dtype=np.float64) for n in co}
    X1, Y1, Z1 = (lambda i: d["dx1"][i + 1]), (lambda j: d["dy1"][j]), (lambda k: d["dzn"][k + 1])
    cn1 = lambda i, j, k: d["cn1"][i - 1, j - 1, k - 1]
    c1d = {n: (lambda arr: (lambda q: arr[q - 1]))(d[n]) for n in ("cn2l", "cn2s", "cn3l", "cn3s", "cn4l", "cn4s")}
    c2l, c2s, c3l, c3s, c4l, c4s = (c1d[n] for n in ("cn2l", "cn2s", "cn3l", "cn3s", "cn4l", "cn4s"))
    area = sum(X1(i) * Y1(j) * Z1(k) for i in range(1, im + 1) for j in range(1, jm + 1) for k in range(1, km + 1))

    def bp2(A):  # boundp.f95:5-21 transposed
        for i in range(0, im + 2):
            for j in range(0, jm + 2):
                A[i, j, km] += A[i, j, km + 1]
                A[i, j, km + 1] = 0.0
                A[i, j, 1] += A[i, j, 0]
                A[i, j, 0] = 0.0

    def bp1(A):  # boundp.f95:23-44 transposed (its j loop first)
        for k in range(0, km + 2):
            for i in range(0, im + 2):
                A[i, 1, k] += A[i, jm + 1, k]
                A[i, jm + 1, k] = 0.0
                A[i, jm, k] += A[i, 0, k]
                A[i, 0, k] = 0.0
        for k in range(0, km + 2):
            for j in range(0, jm + 2):
                A[im, j, k] += A[im + 1, j, k]
                A[im + 1, j, k] = 0.0
                A[1, j, k] += A[0, j, k]
                A[0, j, k] = 0.0

    def meansub(A):  # x -= (sum w x)/W transposed: x_c -= w_c (sum x)/W
        s = float(A[(1, im), (1, jm), (1, km)].sum())
        for i in range(1, im + 1):
            for j in range(1, jm + 1):
                for k in range(1, km + 1):
                    A[i, j, k] -= X1(i) * Y1(j) * Z1(k) * s / area

    bp2(P)
    bp1(P)
    meansub(P)
    for _ in range(niter):
        bp2(P)
        for nrd in (1, 0):
            bp1(P)
            inn = P.arr.copy()
            I0 = FA("p", ip, jp, kp, inn)
            sw = lambda i, j, k: (i + j + k + nrd) % 2 == 1
            fr = lambda i, j, k, c: omega * cn1(i, j, k) * c * I0[i, j, k]
            for i in range(1, im + 1):
                for j in range(1, jm + 1):
                    for k in range(1, km + 1):
                        v = I0[i, j, k]
                        if sw(i, j, k):
                            R[i, j, k] -= omega * cn1(i, j, k) * v
                            P[i, j, k] = (1.0 - omega) * v
                        else:
                            r = v
                            if i > 1: r += fr(i - 1, j, k, c2l(i - 1))
                            if i < im: r += fr(i + 1, j, k, c2s(i + 1))
                            if j > 1: r += fr(i, j - 1, k, c3l(j - 1))
                            if j < jm: r += fr(i, j + 1, k, c3s(j + 1))
                            if k > 1: r += fr(i, j, k - 1, c4l(k - 1))
                            if k < km: r += fr(i, j, k + 1, c4s(k + 1))
                            P[i, j, k] = r
            for j in range(1, jm + 1):
                for k in range(1, km + 1):
                    if sw(1, j, k): P[0, j, k] += fr(1, j, k, c2s(1))
                    if sw(im, j, k): P[im + 1, j, k] += fr(im, j, k, c2l(im))
            for i in range(1, im + 1):
                for k in range(1, km + 1):
                    if sw(i, 1, k): P[i, 0, k] += fr(i, 1, k, c3s(1))
                    if sw(i, jm, k): P[i, jm + 1, k] += fr(i, jm, k, c3l(jm))
                for j in range(1, jm + 1):
                    if sw(i, j, 1): P[i, j, 0] += fr(i, j, 1, c4s(1))
                    if sw(i, j, km): P[i, j, km + 1] += fr(i, j, km, c4l(km))
    meansub(R)
    for i in range(0, im + 1):
        for j in range(0, jm + 1):
            for k in range(0, km + 1):
                rb = lambda a, b, c: R[a, b, c]
                if j >= 1 and k >= 1:
                    x = (rb(i, j, k) / X1(i) if i >= 1 else 0.0) - (rb(i + 1, j, k) / X1(i + 1) if i < im else 0.0)
                    Fb[i, j, k] += x
                    Ub[i, j, k] += x / dt
                if i >= 1 and k >= 1:
                    x = (rb(i, j, k) / Y1(j) if j >= 1 else 0.0) - (rb(i, j + 1, k) / Y1(j + 1) if j < jm else 0.0)
                    Gb[i, j, k] += x
                    Vb[i, j, k] += x / dt
                if i >= 1 and j >= 1:
                    x = (rb(i, j, k) / Z1(k) if k >= 1 else 0.0) - (rb(i, j, k + 1) / Z1(k + 1) if k < km else 0.0)
                    Hb[i, j, k] += x
                    Wb[i, j, k] += x / dt
    R[(1, im), (1, jm), (1, km)] = 0.0
    # bondFG.f95:15-31 transposed
    Fb[1, (1, jm), (1, km)] += Fb[0, (1, jm), (1, km)]
    Fb[0, (1, jm), (1, km)] = 0.0
    Gb[(1, im), jm, (1, km)] += Gb[(1, im), 0, (1, km)]
    Gb[(1, im), 0, (1, km)] = 0.0
    Hb[(1, im), (1, jm), km] = 0.0
    Hb[(1, im), (1, jm), 0] = 0.0
    return (R.arr, P.arr, Fb.arr, Gb.arr, Hb.arr), (Ub.arr, Vb.arr, Wb.arr)


def les_b(ip, jp, kp, co, diu, smb, fb, gb, hb):
    """les.f95:31-182 at the state diu[1..9] (the sm it computes, boundsm,
    the viscous terms added to f, g, h).  co: dx1, dy1, dzn.  Takes the
    adjoints of the outputs sm, f, g, h; returns that of the input sm (0
    where les overwrites it) and those of diu1..9; f, g, h keep theirs.  No
    derivative passes through sqrt where the strain invariant is 0."""
    im, jm, km = ip, jp, kp
    D = {n: FA(f"diu{n}", ip, jp, kp, np.asarray(diu[n], dtype=np.float64)) for n in range(1, 10)}
    Db = {n: FA(f"diu{n}", ip, jp, kp) for n in range(1, 10)}
    Sb = FA("sm", ip, jp, kp, np.asarray(smb, dtype=np.float64).copy())
    sm = FA("sm", ip, jp, kp)
    seed = {c: FA("f", ip, jp, kp, np.asarray(a, dtype=np.float64)) for c, a in (("f", fb), ("g", gb), ("h", hb))}
    d = {n: np.asarray(co[n], dtype=np.float64) for n in ("dx1", "dy1", "dzn")}
    X, Y, Z = (lambda i: d["dx1"][i + 1]), (lambda j: d["dy1"][j]), (lambda k: d["dzn"][k + 1])
    smc = lambda k: (0.1 * (X(0) * Y(0) * Z(k)) ** (1.0 / 3.0)) ** 2

    def grads(i, j, k):
        g = lambda n, a, b, c: D[n][a, b, c]
        return dict(
            d1=g(1, i, j, k), d5=g(5, i, j, k), d9=g(9, i, j, k),
            uy=(g(2, i - 1, j, k) + g(2, i - 1, j + 1, k) + g(2, i, j, k) + g(2, i, j + 1, k)) * 0.25,
            uz=(g(3, i - 1, j, k) + g(3, i - 1, j, k + 1) + g(3, i, j, k) + g(3, i, j, k + 1)) * 0.25,
            vx=(g(4, i, j, k) + g(4, i, j - 1, k) + g(4, i + 1, j, k) + g(4, i + 1, j - 1, k)) * 0.25,
            vz=(g(6, i, j - 1, k) + g(6, i, j - 1, k + 1) + g(6, i, j, k) + g(6, i, j, k + 1)) * 0.25,
            wx=(g(7, i, j, k) + g(7, i, j, k - 1) + g(7, i + 1, j, k) + g(7, i + 1, j, k - 1)) * 0.25,
            wy=(g(8, i, j, k) + g(8, i, j, k - 1) + g(8, i, j + 1, k) + g(8, i, j + 1, k - 1)) * 0.25)

    def inv(gr):
        a, b, c = gr["uy"] + gr["vx"], gr["wy"] + gr["vz"], gr["uz"] + gr["wx"]
        return 2 * (gr["d1"] ** 2 + gr["d5"] ** 2 + gr["d9"] ** 2) + a * a + b * b + c * c, a, b, c

    # the forward's sm (les.f95:132-152) and boundsm (boundsm.f95:13-32)
    for i in range(1, im + 1):
        for j in range(1, jm + 1):
            for k in range(1, km + 1):
                sm[i, j, k] = smc(k) * np.sqrt(inv(grads(i, j, k))[0])
    for k in range(0, km + 2):
        for j in range(-1, jm + 2):
            sm[0, j, k] = sm[1, j, k]
            sm[im + 1, j, k] = sm[im, j, k]
    for k in range(0, km + 2):
        for i in range(0, im + 2):
            sm[i, jm + 1, k] = sm[i, jm, k]
            sm[i, 0, k] = sm[i, 1, k]
    for j in range(-1, jm + 2):
        for i in range(0, im + 2):
            sm[i, j, 0] = -sm[i, j, 1]
            sm[i, j, km + 1] = sm[i, j, km]

    def avg(inner, p, outer, q0, A, B, Sd, i, j, k):
        dd = X if inner == "x" else Y
        win, Sin = (dd(p + 1), dd(p)), dd(p) + dd(p + 1)
        pts = []
        for o, wo in ((0, A), (1, B)):
            for t, wi in ((0, win[0]), (1, win[1])):
                ii, jj, kk = i, j, k
                if inner == "x":
                    ii = p + t
                else:
                    jj = p + t
                if outer == "y":
                    jj = q0 + o
                else:
                    kk = q0 + o
                pts.append(((ii, jj, kk), wo * wi / Sin / Sd))
        return pts

    def terms(i, j, k):  # (component, sign, divisor, evs points, D entries) of les.f95:170-274
        Yjs, Zks, Zkm = Y(j) + Y(j + 1), Z(k) + Z(k + 1), Z(k - 1) + Z(k)
        yield "f", 1, X(i), [((i + 1, j, k), 1.0)], [(1, (i + 1, j, k), 2.0)]
        yield "f", -1, X(i), [((i, j, k), 1.0)], [(1, (i, j, k), 2.0)]
        yield "f", 1, Y(j), avg("x", i, "y", j, Y(j + 1), Y(j), Yjs, i, j, k), [(2, (i, j + 1, k), 1.0), (4, (i + 1, j, k), 1.0)]
        yield "f", -1, Y(j), avg("x", i, "y", j - 1, Y(j + 1), Y(j), Yjs, i, j, k), [(2, (i, j, k), 1.0), (4, (i + 1, j - 1, k), 1.0)]
        yield "f", 1, Z(k), avg("x", i, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(3, (i, j, k + 1), 1.0), (7, (i + 1, j, k), 1.0)]
        yield "f", -1, Z(k), avg("x", i, "z", k - 1, Z(k), Z(k - 1), Zkm, i, j, k), [(3, (i, j, k), 1.0), (7, (i + 1, j, k - 1), 1.0)]
        yield "g", 1, X(i), avg("x", i, "y", j, Y(j + 1), Y(j), Yjs, i, j, k), [(2, (i, j + 1, k), 1.0), (4, (i + 1, j, k), 1.0)]
        yield "g", -1, X(i), avg("x", i - 1, "y", j, Y(j + 1), Y(j), Yjs, i, j, k), [(2, (i - 1, j + 1, k), 1.0), (4, (i, j, k), 1.0)]
        yield "g", 1, Y(j), [((i, j + 1, k), 1.0)], [(5, (i, j + 1, k), 2.0)]
        yield "g", -1, Y(j), [((i, j, k), 1.0)], [(5, (i, j, k), 2.0)]
        yield "g", 1, Z(k), avg("x", i, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(6, (i, j, k + 1), 1.0), (8, (i, j + 1, k), 1.0)]
        yield "g", -1, Z(k), avg("x", i, "z", k - 1, Z(k), Z(k - 1), Zkm, i, j, k), [(6, (i, j, k), 1.0), (8, (i, j + 1, k - 1), 1.0)]
        yield "h", 1, X(i), avg("x", i, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(3, (i, j, k + 1), 1.0), (7, (i + 1, j, k), 1.0)]
        yield "h", -1, X(i), avg("x", i - 1, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(3, (i - 1, j, k + 1), 1.0), (7, (i, j, k), 1.0)]
        yield "h", 1, Y(j), avg("y", j, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(6, (i, j, k + 1), 1.0), (8, (i, j + 1, k), 1.0)]
        yield "h", -1, Y(j), avg("y", j - 1, "z", k, Z(k + 1), Z(k), Zks, i, j, k), [(6, (i, j - 1, k + 1), 1.0), (8, (i, j, k), 1.0)]
        yield "h", 1, Z(k), [((i, j, k + 1), 1.0)], [(9, (i, j, k + 1), 2.0)]
        yield "h", -1, Z(k), [((i, j, k), 1.0)], [(9, (i, j, k), 2.0)]

    for i in range(1, im + 1):
        for j in range(1, jm + 1):
            for k in range(1, km + 1):
                for comp, sgn, div, pts, dl in terms(i, j, k):
                    vb = sgn * seed[comp][i, j, k] / div
                    evs = sum(w * sm[p] for p, w in pts)
                    Dv = sum(fac * D[n][loc] for n, loc, fac in dl)
                    for p, w in pts:
                        Sb[p] += vb * Dv * w
                    for n, loc, fac in dl:
                        Db[n][loc] += vb * evs * fac
    # boundsm transposed, its three loops last first
    for j in range(-1, jm + 2):
        for i in range(0, im + 2):
            Sb[i, j, km] += Sb[i, j, km + 1]
            Sb[i, j, km + 1] = 0.0
            Sb[i, j, 1] -= Sb[i, j, 0]
            Sb[i, j, 0] = 0.0
    for k in range(0, km + 2):
        for i in range(0, im + 2):
            Sb[i, 1, k] += Sb[i, 0, k]
            Sb[i, 0, k] = 0.0
            Sb[i, jm, k] += Sb[i, jm + 1, k]
            Sb[i, jm + 1, k] = 0.0
    for k in range(0, km + 2):
        for j in range(-1, jm + 2):
            Sb[im, j, k] += Sb[im + 1, j, k]
            Sb[im + 1, j, k] = 0.0
            Sb[1, j, k] += Sb[0, j, k]
            Sb[0, j, k] = 0.0
    # sm = smc(k) sqrt(Q) transposed
    for i in range(1, im + 1):
        for j in range(1, jm + 1):
            for k in range(1, km + 1):
                b0 = Sb[i, j, k]
                Sb[i, j, k] = 0.0
                gr = grads(i, j, k)
                q, a, b, c = inv(gr)
                if not q > 0.0:
                    continue
                qb = b0 * smc(k) * 0.5 / np.sqrt(q)
                for n, key in ((1, "d1"), (5, "d5"), (9, "d9")):
                    Db[n][i, j, k] += qb * 4.0 * gr[key]
                ab, bb, cb = 0.5 * a * qb, 0.5 * b * qb, 0.5 * c * qb
                for n, val, pts in (
                        (2, ab, ((i - 1, j, k), (i - 1, j + 1, k), (i, j, k), (i, j + 1, k))),
                        (4, ab, ((i, j, k), (i, j - 1, k), (i + 1, j, k), (i + 1, j - 1, k))),
                        (3, cb, ((i - 1, j, k), (i - 1, j, k + 1), (i, j, k), (i, j, k + 1))),
                        (7, cb, ((i, j, k), (i, j, k - 1), (i + 1, j, k), (i + 1, j, k - 1))),
                        (6, bb, ((i, j - 1, k), (i, j - 1, k + 1), (i, j, k), (i, j, k + 1))),
                        (8, bb, ((i, j, k), (i, j, k - 1), (i, j + 1, k), (i, j + 1, k - 1)))):
                    for p in pts:
                        Db[n][p] += val
    return Sb.arr, {n: Db[n].arr for n in range(1, 10)}


# ---- one whole time step (the sequence of oracle_run_steps, main_ocl.f95:
# 264-299, with the external inflow profile) and its reference adjoint

STATE = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold", "rhs", "sm"]
_WORK = [f"{a}{n}" for n in range(1, 10) for a in ("nou", "diu", "cov")] + ["dfu1", "dfv1", "dfw1"]


class Step64:
    """One step of the FP64 oracle with niter SOR iterations (no stop test)
    and its adjoint.  co: the case's metrics, masks and Poisson coefficients
    (Fortran layout); prm: dt, ro, vn, alpha, beta, omega.  drag: an optional
    per-column scale s(i, j) (ip x jp) on feedbf's force, f += s fx instead
    of f += fx (feedbf.f95:61-66; s = 1 is the reference)."""

    def __init__(self, ip, jp, kp, co, prm, niter, drag=None):
        from oracle import fp64
        import ctypes as C
        self.ip, self.jp, self.kp, self.prm, self.niter = ip, jp, kp, prm, niter
        self.drag = None if drag is None else np.asarray(drag, dtype=np.float64)
        self.co = {n: np.asfortranarray(np.asarray(a, dtype=np.float64)) for n, a in co.items()}
        L = fp64.lib()
        i, d, p = C.c_int, C.c_double, C.c_void_p
        L.oracle_velnw.argtypes = [i, i, i, p, d, p, p, d, p, p, p, p, p, p, p]
        L.oracle_bondv1_ext_wind_profile.argtypes = [i, p, p, p, p, p, i, i, i, d, p, p]
        L.oracle_velfg.argtypes = [i, i, i] + [p] * 10 + [d] + [p] * 30
        L.oracle_feedbf.argtypes = [i, i, i] + [p] * 9 + [d, d, d] + [p] * 6
        L.oracle_les.argtypes = [i, p, p, p, p, i, i] + [p] * 13
        L.oracle_adam.argtypes = [i, i, p, i, i, i, p, p, p, p, p]
        L.oracle_press_ex.argtypes = [i, i, i] + [p] * 10 + [d] + [p] * 8 + [i, d, d, p, p, p]
        L.oracle_press_ex.restype = C.c_int
        self.L = L

    def forward(self, n, state, wp):
        """The step from state (dict of STATE arrays) and inflow wp(j, k);
        returns the new state and the forward values the adjoint reads."""
        ip, jp, kp, L, pr, c = self.ip, self.jp, self.kp, self.L, self.prm, self.co
        a = {k: np.asfortranarray(np.array(state[k], dtype=np.float64)) for k in STATE}
        P = lambda x: x.ctypes.data
        wpa = np.asfortranarray(np.array(wp, dtype=np.float64))
        L.oracle_velnw(kp, jp, ip, P(a["p"]), pr["ro"], P(c["dxs"]), P(a["u"]), pr["dt"], P(a["f"]), P(c["dys"]),
                       P(a["v"]), P(a["g"]), P(c["dzs"]), P(a["w"]), P(a["h"]))
        tape = {"uvw_velnw": {k: a[k].copy() for k in ("u", "v", "w")}}
        L.oracle_bondv1_ext_wind_profile(jp, P(a["u"]), P(c["z2"]), P(c["dzn"]), P(a["v"]), P(a["w"]), kp, n, ip,
                                         pr["dt"], P(c["dxs"]), P(wpa))
        tape["uvw_bondv1"] = {k: a[k].copy() for k in ("u", "v", "w")}
        s = {k: np.asfortranarray(np.zeros(FL.alloc(k, ip, jp, kp).shape)) for k in _WORK}
        s.update({k: np.asfortranarray(np.zeros(FL.alloc("f", ip, jp, kp).shape)) for k in ("fx", "fy", "fz")})
        A = lambda k: P(a[k]) if k in a else (P(s[k]) if k in s else P(c[k]))
        L.oracle_velfg(kp, jp, ip, *[A(k) for k in ("dx1", "cov1", "cov2", "cov3", "dfu1", "diu1", "diu2", "dy1",
                                                    "diu3", "dzn")], pr["vn"],
                       *[A(k) for k in ("f", "cov4", "cov5", "cov6", "dfv1", "diu4", "diu5", "diu6", "g", "cov7",
                                        "cov8", "cov9", "dfw1", "diu7", "diu8", "diu9", "dzs", "h", "nou1", "u",
                                        "nou5", "v", "nou9", "w", "nou2", "nou3", "nou4", "nou6", "nou7", "nou8")])
        tape["diu"] = {m: s[f"diu{m}"].copy() for m in range(1, 10)}
        f0 = {k: a[k].copy() for k in ("f", "g", "h")}
        L.oracle_feedbf(kp, jp, ip, A("usum"), A("u"), A("bmask1"), A("vsum"), A("v"), A("cmask1"), A("wsum"),
                        A("w"), A("dmask1"), pr["alpha"], pr["dt"], pr["beta"], A("fx"), A("fy"), A("fz"),
                        A("f"), A("g"), A("h"))
        tape["fxyz"] = [s[k].copy() for k in ("fx", "fy", "fz")]
        if self.drag is not None:  # f = f0 + s fx on the interior
            for k, x in zip(("f", "g", "h"), ("fx", "fy", "fz")):
                F, F0, X = (FA("f", ip, jp, kp, arr) for arr in (a[k], f0[k], s[x]))
                F[(1, ip), (1, jp), (1, kp)] = F0[(1, ip), (1, jp), (1, kp)] + \
                    self.drag[:, :, np.newaxis] * X[(1, ip), (1, jp), (1, kp)]
        delx1 = np.zeros(kp)
        L.oracle_les(kp, P(delx1), A("dx1"), A("dy1"), A("dzn"), jp, ip, *[A(f"diu{m}") for m in range(1, 10)],
                     A("sm"), A("f"), A("g"), A("h"))
        L.oracle_adam(n, 1 << 20, A("fold"), ip, jp, kp, A("gold"), A("hold"), A("f"), A("g"), A("h"))
        it = L.oracle_press_ex(kp, jp, ip, A("rhs"), A("u"), A("dx1"), A("v"), A("dy1"), A("w"), A("dzn"), A("f"),
                               A("g"), A("h"), pr["dt"], A("cn1"), A("cn2l"), A("p"), A("cn2s"), A("cn3l"),
                               A("cn3s"), A("cn4l"), A("cn4s"), self.niter, -1.0, pr["omega"], None, None, None)
        assert it == self.niter
        return a, tape

    def adjoint(self, n, tape, wp, seeds):
        """Adjoints of the step's inputs (STATE arrays) from those of its
        outputs (seeds), at the forward values in tape, and the gradients of
        the parameters: {"wp": inflow profile, "drag": drag scale or None}."""
        ip, jp, kp, pr, c = self.ip, self.jp, self.kp, self.prm, self.co
        b = {k: np.array(seeds[k], dtype=np.float64) for k in STATE}
        # press (press.f95:49-146)
        (b["rhs"], b["p"], b["f"], b["g"], b["h"]), uvw = press_b(
            ip, jp, kp, c, pr["dt"], pr["omega"], self.niter, b["rhs"], b["p"], b["f"], b["g"], b["h"])
        for k, x in zip(("u", "v", "w"), uvw):
            b[k] += x
        # adam
        (b["f"], b["fold"]), (b["g"], b["gold"]), (b["h"], b["hold"]) = adam_b(
            ip, jp, kp, b["f"], b["g"], b["h"], b["fold"], b["gold"], b["hold"])
        # les (diu from velfg)
        b["sm"], diub = les_b(ip, jp, kp, c, tape["diu"], b["sm"], b["f"], b["g"], b["h"])
        # feedbf (with the drag scale, fx's adjoint is s times f's)
        xb = [b["f"], b["g"], b["h"]]
        dragb = None
        if self.drag is not None:
            dragb = np.zeros((ip, jp))
            for q, k in enumerate(("f", "g", "h")):
                B, X = FA("f", ip, jp, kp, b[k]), FA("f", ip, jp, kp, tape["fxyz"][q])
                dragb += np.sum(X[(1, ip), (1, jp), (1, kp)] * B[(1, ip), (1, jp), (1, kp)], axis=2)
                xs = b[k].copy()
                XS = FA("f", ip, jp, kp, xs)
                XS[(1, ip), (1, jp), (1, kp)] = self.drag[:, :, np.newaxis] * B[(1, ip), (1, jp), (1, kp)]
                xb[q] = xs
        (b["usum"], b["vsum"], b["wsum"]), uvw = feedbf_b(ip, jp, kp, c, pr["alpha"], pr["dt"], pr["beta"],
                                                          b["usum"], b["vsum"], b["wsum"], *xb)
        for k, x in zip(("u", "v", "w"), uvw):
            b[k] += x
        # velfg at the state after bondv1; it overwrites f, g (k = 1..km) and h (k = 1..km-1)
        t = tape["uvw_bondv1"]
        uvw, _ = velfg_b(ip, jp, kp, c, pr["vn"], t["u"], t["v"], t["w"], b["f"], b["g"], b["h"], diub)
        for k, x in zip(("u", "v", "w"), uvw):
            b[k] += x
        for k, kr in (("f", (1, kp)), ("g", (1, kp)), ("h", (1, kp - 1))):
            A = FA("f", ip, jp, kp, b[k])
            A[(1, ip), (1, jp), kr] = 0.0
        # bondv1 (external inflow) at the state after velnw
        t = tape["uvw_velnw"]
        b["u"], b["v"], b["w"], wpb = bondv1_ext_b(ip, jp, kp, c["dxs"], pr["dt"], n, wp, t["u"], t["v"], t["w"],
                                                   b["u"], b["v"], b["w"])
        # velnw
        pb, fb, gb, hb = velnw_b(ip, jp, kp, c["dxs"], c["dys"], c["dzs"], pr["ro"], pr["dt"], b["u"], b["v"],
                                 b["w"])
        for k, x in (("p", pb), ("f", fb), ("g", gb), ("h", hb)):
            b[k] += x
        return b, {"wp": wpb, "drag": dragb}


# ---- the config-3 style objective: time- and box-mean resolved TKE with the
# cell-centred velocities of anime.f95:45-47, and its gradient by the step
# adjoint with checkpoints and recomputation

def tke(ip, jp, kp, state, box):
    """Mean over the cells of box ((i0, i1), (j0, j1), (k0, k1), inclusive)
    of 0.5 (uc^2 + vc^2 + wc^2), uc = 0.5 (u(i-1) + u(i)) and alike."""
    (i0, i1), (j0, j1), (k0, k1) = box
    U, V, W = (FA(n, ip, jp, kp, np.asarray(state[n], dtype=np.float64)) for n in ("u", "v", "w"))
    I, J, K = (i0, i1), (j0, j1), (k0, k1)
    sh = lambda r, d: (r[0] + d, r[1] + d)
    uc = 0.5 * (U[sh(I, -1), J, K] + U[I, J, K])
    vc = 0.5 * (V[I, sh(J, -1), K] + V[I, J, K])
    wc = 0.5 * (W[I, J, sh(K, -1)] + W[I, J, K])
    return float(np.mean(0.5 * (uc * uc + vc * vc + wc * wc)))


def tke_seed(ip, jp, kp, state, box, scale, bar):
    """bar[u, v, w] += scale * d tke / d (u, v, w) at state."""
    (i0, i1), (j0, j1), (k0, k1) = box
    ncell = (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1)
    I, J, K = (i0, i1), (j0, j1), (k0, k1)
    sh = lambda r, d: (r[0] + d, r[1] + d)
    for n, lower in (("u", (sh(I, -1), J, K)), ("v", (I, sh(J, -1), K)), ("w", (I, J, sh(K, -1)))):
        X = FA(n, ip, jp, kp, np.asarray(state[n], dtype=np.float64))
        B = FA(n, ip, jp, kp, bar[n])
        c = 0.5 * (X[lower] + X[I, J, K])  # the centred value
        g = scale / ncell * 0.5 * c  # d(0.5 c^2)/dc * dc/dx, for each of the two x
        B[lower] += g
        B[I, J, K] += g


def tke_gradient(step, n0, nt, state0, wp, box, ckpt):
    """J = (1/nt) sum over steps n0 .. n0+nt-1 of tke after the step, and its
    gradients with respect to the inflow profile wp (held over the steps),
    the drag scale (when the step has one) and the initial state, by the
    step adjoint in reverse.  Only every ckpt-th
    state is kept; each segment's forward values are recomputed from its
    checkpoint before the segment is reversed."""
    ip, jp, kp = step.ip, step.jp, step.kp
    ckpts, s, J = {0: state0}, state0, 0.0
    for t in range(nt):
        s, _ = step.forward(n0 + t, s, wp)
        J += tke(ip, jp, kp, s, box) / nt
        if (t + 1) % ckpt == 0 and t + 1 < nt:
            ckpts[t + 1] = s
    bar = {k: np.zeros(FL.alloc(k, ip, jp, kp).shape) for k in STATE}
    grads = {"wp": np.zeros(np.asarray(wp).shape), "drag": None if step.drag is None else np.zeros((ip, jp))}
    for t0 in sorted(ckpts, reverse=True):
        t1 = min(t0 + ckpt, nt)
        s, seg = ckpts[t0], []
        for t in range(t0, t1):
            out, tape = step.forward(n0 + t, s, wp)
            seg.append((tape, out))
            s = out
        for t in reversed(range(t0, t1)):
            tape, out = seg[t - t0]
            tke_seed(ip, jp, kp, out, box, 1.0 / nt, bar)
            bar, g = step.adjoint(n0 + t, tape, wp, bar)
            grads["wp"] += g["wp"]
            if grads["drag"] is not None:
                grads["drag"] += g["drag"]
    return J, grads, bar
