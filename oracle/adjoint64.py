"""FP64 reference adjoints (reverse mode) for routines whose CUDA adjoint is
still to come, in vectorised NumPy.

TEST INFRASTRUCTURE ONLY, like the rest of oracle/: the reference gradient
that the CUDA adjoint entries are checked against, itself checked against
central differences of the FP64 oracle (oracle/fp64.py) in
tests/test_adjoint64.py.

bondv1_ext_b: bondv1_ext_wind_profile.f95:27-127 (inflow from the external
profile, n == 1 broadcast, outflow with uout, periodic, top and ground).

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
