// les_adjstep.cuh -- reverse-mode kernels of the routines whose adjoint
// les_adjoint.cuh does not hold (vel2 + velfg, bondv1 with the external
// inflow profile), and of the pieces the adjoint of a whole time step adds
// (the drag-scale gradient, the TKE objective and its seed).  All in FP32
// with the forward values recomputed from the step's input state;
// accumulations that cross cells use atomic adds, parameter gradients FP64.
#pragma once

#include "les_adjoint.cuh"

namespace les {
namespace {

// ---- vel2.f95:48-188 + velFG.f95:56-105 transposed -------------------------
// velfg reads u, v, w through 27 face arrays: nou_n (an interpolant), diu_n
// (a difference quotient) and cov_n = nou_n * diu_n (cov4/cov7 subtract
// u0 = 0), n = 1..9, computed on ranges and then copied onto boundary faces
// (vel2.f95:125-188); f, g, h are sums of cov and diu values of the cell's
// faces (velFG.f95:56-105).  Its adjoint at the forward (u, v, w) runs the
// three stages backwards: the velfg sums scatter into the face adjoints,
// the boundary copies move their adjoints back to the sources (statement by
// statement, last first), and every computed face sends
//     nou_b += cov_b * diu,  diu_b += cov_b * nou
// through its interpolation and difference weights to u, v, w.  diu_b starts
// as what les's adjoint produced (les reads diu).
struct VelfgB {
    Geo g;
    UVW q;                  // forward u, v, w (after bondv1)
    float vn;
    const float *fb, *gb, *hb;
    float *nb[9], *db[9], *cb[9];  // face adjoints, box layout
    float *ub, *vb, *wb;    // accumulate
};

__device__ __forceinline__ void aadd(float *a, const Geo &g, int i, int j, int k, float v) {
    atomicAdd(&a[IX(g, i, j, k)], v);
}

// Stage 1: velFG.f95:56-105 transposed, per cell (i, j, k) of I x J x K.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adjv_fgh(VelfgB A) {
    const Geo &g = A.g;
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    const float X0 = g.dx1[i], X1 = g.dx1[i + 1], Y0 = g.dy1[j], Y1 = g.dy1[j + 1];
    const float Zn0 = g.dzn[k], Zn1 = g.dzn[k + 1], Zs0 = g.dzs[k];
    {  // f: -(cov1 x-average + cov2, cov3 pair means) + vn (diu1, diu2, diu3 differences)
        const float s = -A.fb[c], d = A.vn * A.fb[c], sx = X0 + X1;
        aadd(A.cb[0], g, i, j, k, s * X1 / sx);
        aadd(A.cb[0], g, i + 1, j, k, s * X0 / sx);
        aadd(A.cb[1], g, i, j, k, s / 2.0f);
        aadd(A.cb[1], g, i, j + 1, k, s / 2.0f);
        aadd(A.cb[2], g, i, j, k, s / 2.0f);
        aadd(A.cb[2], g, i, j, k + 1, s / 2.0f);
        aadd(A.db[0], g, i, j, k, -2.0f * d / sx);
        aadd(A.db[0], g, i + 1, j, k, 2.0f * d / sx);
        aadd(A.db[1], g, i, j, k, -d / Y0);
        aadd(A.db[1], g, i, j + 1, k, d / Y0);
        aadd(A.db[2], g, i, j, k, -d / Zn0);
        aadd(A.db[2], g, i, j, k + 1, d / Zn0);
    }
    {  // g
        const float s = -A.gb[c], d = A.vn * A.gb[c], sy = Y0 + Y1;
        aadd(A.cb[3], g, i, j, k, s / 2.0f);
        aadd(A.cb[3], g, i + 1, j, k, s / 2.0f);
        aadd(A.cb[4], g, i, j, k, s * Y1 / sy);
        aadd(A.cb[4], g, i, j + 1, k, s * Y0 / sy);
        aadd(A.cb[5], g, i, j, k, s / 2.0f);
        aadd(A.cb[5], g, i, j, k + 1, s / 2.0f);
        aadd(A.db[3], g, i, j, k, -d / X0);
        aadd(A.db[3], g, i + 1, j, k, d / X0);
        aadd(A.db[4], g, i, j, k, -2.0f * d / sy);
        aadd(A.db[4], g, i, j + 1, k, 2.0f * d / sy);
        aadd(A.db[5], g, i, j, k, -d / Zn0);
        aadd(A.db[5], g, i, j, k + 1, d / Zn0);
    }
    if (k <= g.km - 1) {  // h (k = 1..km-1)
        const float s = -A.hb[c], d = A.vn * A.hb[c], sz = Zn0 + Zn1;
        aadd(A.cb[6], g, i, j, k, s / 2.0f);
        aadd(A.cb[6], g, i + 1, j, k, s / 2.0f);
        aadd(A.cb[7], g, i, j, k, s / 2.0f);
        aadd(A.cb[7], g, i, j + 1, k, s / 2.0f);
        aadd(A.cb[8], g, i, j, k, s * Zn1 / sz);
        aadd(A.cb[8], g, i, j, k + 1, s * Zn0 / sz);
        aadd(A.db[6], g, i, j, k, -d / X0);
        aadd(A.db[6], g, i + 1, j, k, d / X0);
        aadd(A.db[7], g, i, j, k, -d / Y0);
        aadd(A.db[7], g, i, j + 1, k, d / Y0);
        aadd(A.db[8], g, i, j, k, -d / Zs0);
        aadd(A.db[8], g, i, j, k + 1, d / Zs0);
    }
}

// a[src] += a[dst]; a[dst] = 0 (one copy dst = src of vel2 transposed).
__device__ __forceinline__ void amv(float *a, const Geo &g, int di, int dj, int dk, int si, int sj, int sk) {
    float &d = a[IX(g, di, dj, dk)];
    a[IX(g, si, sj, sk)] += d;
    d = 0.0f;
}

// Stage 2a, the last copies of vel2.f95:177-188 transposed (they read the
// arrays the later stage-2b copies write, so they go back first):
// diu6, diu4 (i, 0, k) = (i, jm, k) for i 1..im+1, k 1..km+1 and
// diu3, diu2 (im+1, j, k) = (im, j, k) for j 1..jm+1, k 1..km+1.
__global__ void k_adjv_copies_a(VelfgB A) {
    const Geo &g = A.g;
    const int im = g.im, jm = g.jm, km = g.km;
    const int nA = (im + 1) * (km + 1), nB = (jm + 1) * (km + 1);
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nA) {
        const int i = 1 + t % (im + 1), k = 1 + t / (im + 1);
        amv(A.db[5], g, i, 0, k, i, jm, k);
        amv(A.db[3], g, i, 0, k, i, jm, k);
    } else if ((t -= nA) < nB) {
        const int j = 1 + t % (jm + 1), k = 1 + t / (jm + 1);
        amv(A.db[2], g, im + 1, j, k, im, j, k);
        amv(A.db[1], g, im + 1, j, k, im, j, k);
    }
}

// Stage 2b, vel2.f95:125-176 transposed: the j-periodic copies of the n = 8,
// 5, 2 groups (x(i,0,k) = x(i,jm,k), x(i,jm+1,k) = x(i,1,k)) and the i copies
// x(im+1,j,k) = x(im,j,k) of the n = 7, 4, 1 groups, for nou, diu and cov.
// Every array is touched by one of these loops only.
__global__ void k_adjv_copies_b(VelfgB A) {
    const Geo &g = A.g;
    const int im = g.im, jm = g.jm, km = g.km;
    const int nJ = im * km, nI = jm * km;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int grp = t / (nJ + nI);  // 0: n = 8 and 7, 1: n = 5 and 4, 2: n = 2 and 1
    if (grp > 2) return;
    t -= grp * (nJ + nI);
    const int nj = grp == 0 ? 7 : (grp == 1 ? 4 : 1);  // zero-based index of the j-copied group
    const int ni = nj - 1;                              // and of the i-copied group
    const int kmax = grp == 0 ? km - 1 : km;
    float *arr_j[3] = {A.cb[nj], A.db[nj], A.nb[nj]}, *arr_i[3] = {A.cb[ni], A.db[ni], A.nb[ni]};
    if (t < nJ) {
        const int i = 1 + t % im, k = 1 + t / im;
        if (k > kmax) return;
        for (int a = 0; a < 3; ++a) {
            amv(arr_j[a], g, i, jm + 1, k, i, 1, k);
            amv(arr_j[a], g, i, 0, k, i, jm, k);
        }
    } else {
        t -= nJ;
        const int j = 1 + t % jm, k = 1 + t / jm;
        if (k > kmax) return;
        for (int a = 0; a < 3; ++a) amv(arr_i[a], g, im + 1, j, k, im, j, k);
    }
}

// Stage 3, vel2.f95:48-123 transposed: every face of the computed ranges
// (n = 3, 6 to k = km+1, n = 7, 8 to km-1) sends its adjoint to u, v, w.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adjv_faces(VelfgB A) {
    const Geo &g = A.g;
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    const int im = g.im, jm = g.jm, km = g.km;
    if (i > im || j > jm) return;
    const UVW &q = A.q;
    const int c = IX(g, i, j, k);
    const float X0 = g.dx1[i], X1 = g.dx1[i + 1], Xm = g.dx1[i - 1];
    const float Y0 = g.dy1[j], Y1 = g.dy1[j + 1], Ym = g.dy1[j - 1];
    // face n (zero-based) at this cell: a = nou's adjoint, b = diu's
    auto face = [&](int n, float nou, float diu, float &a, float &b) {
        const float cv = A.cb[n][c];
        a = A.nb[n][c] + cv * diu;
        b = A.db[n][c] + cv * nou;
    };
    float a, b;
    if (k <= km) {
        face(0, nou1_raw(g, q, i, j, k), diu1_raw(g, q, i, j, k), a, b);
        aadd(A.ub, g, i - 1, j, k, a / 2.0f - b / X0);
        aadd(A.ub, g, i, j, k, a / 2.0f + b / X0);
        face(4, nou5_raw(g, q, i, j, k), diu5_raw(g, q, i, j, k), a, b);
        aadd(A.vb, g, i, j - 1, k, a / 2.0f - b / Y0);
        aadd(A.vb, g, i, j, k, a / 2.0f + b / Y0);
        const float Zn0 = g.dzn[k];
        face(8, nou9_raw(g, q, i, j, k), diu9_raw(g, q, i, j, k), a, b);
        aadd(A.wb, g, i, j, k - 1, a / 2.0f - b / Zn0);
        aadd(A.wb, g, i, j, k, a / 2.0f + b / Zn0);
        const float sx = X0 + X1, sy = Ym + Y0;
        face(1, nou2_raw(g, q, i, j, k), diu2_raw(g, q, i, j, k), a, b);
        aadd(A.vb, g, i, j - 1, k, a * X1 / sx);
        aadd(A.vb, g, i + 1, j - 1, k, a * X0 / sx);
        aadd(A.ub, g, i, j - 1, k, -2.0f * b / sy);
        aadd(A.ub, g, i, j, k, 2.0f * b / sy);
        const float sy1 = Y0 + Y1, sxm = Xm + X0;
        face(3, nou4_raw(g, q, i, j, k), diu4_raw(g, q, i, j, k), a, b);
        aadd(A.ub, g, i - 1, j, k, a * Y1 / sy1);
        aadd(A.ub, g, i - 1, j + 1, k, a * Y0 / sy1);
        aadd(A.vb, g, i - 1, j, k, -2.0f * b / sxm);
        aadd(A.vb, g, i, j, k, 2.0f * b / sxm);
        if (k <= km - 1) {
            const float sz = g.dzn[k] + g.dzn[k + 1];
            face(6, nou7_raw(g, q, i, j, k), diu7_raw(g, q, i, j, k), a, b);
            aadd(A.ub, g, i - 1, j, k, a * g.dzn[k + 1] / sz);
            aadd(A.ub, g, i - 1, j, k + 1, a * g.dzn[k] / sz);
            aadd(A.wb, g, i - 1, j, k, -2.0f * b / sxm);
            aadd(A.wb, g, i, j, k, 2.0f * b / sxm);
            face(7, nou8_raw(g, q, i, j, k), diu8_raw(g, q, i, j, k), a, b);
            aadd(A.vb, g, i, j - 1, k, a * g.dzn[k + 1] / sz);
            aadd(A.vb, g, i, j - 1, k + 1, a * g.dzn[k] / sz);
            aadd(A.wb, g, i, j - 1, k, -2.0f * b / sy);
            aadd(A.wb, g, i, j, k, 2.0f * b / sy);
        }
    }
    {  // n = 3, 6: k = 1..km+1, from the plane below
        const float sx = X0 + X1, sy1 = Y0 + Y1, zs = g.dzs[k - 1];
        face(2, nou3_raw(g, q, i, j, k), diu3_raw(g, q, i, j, k), a, b);
        aadd(A.wb, g, i, j, k - 1, a * X1 / sx);
        aadd(A.wb, g, i + 1, j, k - 1, a * X0 / sx);
        aadd(A.ub, g, i, j, k - 1, -b / zs);
        aadd(A.ub, g, i, j, k, b / zs);
        face(5, nou6_raw(g, q, i, j, k), diu6_raw(g, q, i, j, k), a, b);
        aadd(A.wb, g, i, j, k - 1, a * Y1 / sy1);
        aadd(A.wb, g, i, j + 1, k - 1, a * Y0 / sy1);
        aadd(A.vb, g, i, j, k - 1, -b / zs);
        aadd(A.vb, g, i, j, k, b / zs);
    }
}

// velfg overwrites f, g (k = 1..km) and h (k = 1..km-1): their adjoints
// with respect to the previous contents are zero there.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adjv_zero_fgh(Geo g, float *fb, float *gb, float *hb) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    fb[c] = 0.0f;
    gb[c] = 0.0f;
    if (k <= g.km - 1) hb[c] = 0.0f;
}

// ---- bondv1_ext_wind_profile.f95:27-127 transposed ---------------------------
// Forward values it needs, from the state after velnw with the inflow (and
// the n == 1 broadcast) applied -- the state the tail of bondv1 starts from:
// uout's extremes (first in the reference's k-outer, j-inner order, as
// amax1/amin1 keep them) and, for the outflow, the differences across the
// last cell.  Extremes are packed keys: value bits made order-preserving in
// the high word, the k-major index (or its complement, so the first one
// wins a tie under max) in the low word.
struct BondvTape {
    unsigned long long kmax, kmin;  // packed extremes of u(im, 1..jm, 1..km)
    double uoutb;                   // adjoint of uout
    float uout;                     // (max(0, max u) + min(0, min u)) / 2
};
__device__ __forceinline__ unsigned ord_bits(float x) {
    const unsigned b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_value(unsigned o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
__global__ void k_adjb_reset(BondvTape *t) {
    t->kmax = 0ull;
    t->kmin = ~0ull;
    t->uoutb = 0.0;
    t->uout = 0.0f;
}
__global__ void __launch_bounds__(256) k_adjb_extremes(Geo g, const float *u, BondvTape *t) {
    const int n = g.jm * g.km;
    unsigned long long mx = 0ull, mn = ~0ull;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int j = 1 + q % g.jm, k = 1 + q / g.jm;  // q is the k-major position
        const unsigned long long o = ord_bits(u[IX(g, g.im, j, k)]);
        mx = max(mx, (o << 32) | (unsigned)(0xffffffffu - (unsigned)q));
        mn = min(mn, (o << 32) | (unsigned)q);
    }
    for (int off = 16; off >= 1; off >>= 1) {
        mx = max(mx, __shfl_down_sync(0xffffffffu, mx, off));
        mn = min(mn, __shfl_down_sync(0xffffffffu, mn, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&t->kmax, mx);
        atomicMin(&t->kmin, mn);
    }
}
__global__ void k_adjb_uout(BondvTape *t) {
    const float aaa = fmaxf(0.0f, ord_value((unsigned)(t->kmax >> 32)));
    const float bbb = fminf(0.0f, ord_value((unsigned)(t->kmin >> 32)));
    t->uout = (aaa + bbb) / 2.0f;
}

// w's zeroed planes, then top/ground of v and u (bondv1.f95:120-137 with the
// w(-1, j, .) writes that land on w(ip+1, j-1, .)).  stage 0: the w planes;
// stage 1: x(.,.,km) += x(.,.,km+1), x(.,.,1) -= x(.,.,0) for v and u.
__global__ void k_adjb_topground(Geo g, float *ub, float *vb, float *wb, int stage) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int ni = im + 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (stage == 0) {
        if (t >= ni * (jm + 3)) return;
        const int i = t % ni, j = -1 + t / ni;
        wb[IX(g, i, j, 0)] = 0.0f;
        wb[IX(g, i, j, km)] = 0.0f;
        if (i == im + 1 && j <= jm) {  // w(-1, j+1, .)
            wb[IX(g, im + 1, j, 0)] = 0.0f;
            wb[IX(g, im + 1, j, km)] = 0.0f;
        }
        if (i == im + 1 && j == jm + 1) {  // w(-1, -1..., .): the aliased corner
            wb[IX(g, im + 1, jm + 1, -1)] = 0.0f;
            wb[IX(g, im + 1, jm + 1, km - 1)] = 0.0f;
        }
        return;
    }
    if (t >= ni * (jm + 2)) return;
    const int i = t % ni, j = t / ni;
    float *arr[2] = {vb, ub};
    for (int a = 0; a < 2; ++a) {
        float *A = arr[a];
        A[IX(g, i, j, km)] += A[IX(g, i, j, km + 1)];
        A[IX(g, i, j, km + 1)] = 0.0f;
        A[IX(g, i, j, 1)] -= A[IX(g, i, j, 0)];
        A[IX(g, i, j, 0)] = 0.0f;
    }
}

// Periodic j (bondv1.f95:100-117) transposed: w for k = 0..km, v and u for
// k = 0..km+1, i = 0..im+1.
__global__ void k_adjb_periodic(Geo g, float *ub, float *vb, float *wb) {
    const int ni = g.im + 2, nk = g.km + 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ni * nk) return;
    const int i = t % ni, k = t / ni;
    const int jm = g.jm;
    auto per = [&](float *A) {
        A[IX(g, i, 1, k)] += A[IX(g, i, jm + 1, k)];
        A[IX(g, i, jm + 1, k)] = 0.0f;
        A[IX(g, i, jm, k)] += A[IX(g, i, 0, k)];
        A[IX(g, i, 0, k)] = 0.0f;
    };
    if (k <= g.km) per(wb);
    per(vb);
    per(ub);
}

// Outflow (bondv1.f95:81-97) transposed, w then v then u at e = im+1, im+1,
// im: x(e) = x(e) - c (x(e) - x(e-1)), c = dt uout / dxs(im).  The forward
// differences come from the tape state (before the outflow).  Per (j, k);
// the uout adjoint -dt/dxs(im) * sum(dx * ob) is summed in FP64.
__global__ void __launch_bounds__(256) k_adjb_outflow(Geo g, const float *u1, const float *v1, const float *w1,
                                                      float *ub, float *vb, float *wb, BondvTape *t) {
    const int n = g.jm * g.km;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int im = g.im;
    const float ds = g.dxs[im], dt = g.dt;
    const float c = dt * t->uout / ds;
    double acc = 0.0;
    if (q < n) {
        const int j = 1 + q % g.jm, k = 1 + q / g.jm;
        auto out = [&](float *A, const float *X, int e) {
            const float dx = X[IX(g, e, j, k)] - X[IX(g, e - 1, j, k)];
            const float ob = A[IX(g, e, j, k)];
            acc += (double)(-dt / ds * dx * ob);
            A[IX(g, e - 1, j, k)] += c * ob;
            A[IX(g, e, j, k)] = (1.0f - c) * ob;
        };
        out(wb, w1, im + 1);
        out(vb, v1, im + 1);
        out(ub, u1, im);
    }
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&t->uoutb, acc);
}

// uout = (max(0, max u(im)) + min(0, min u(im))) / 2: its adjoint goes half
// to the first maximal and half to the first minimal element (when the
// extreme is not clipped at 0).
__global__ void k_adjb_uout_b(Geo g, float *ub, const BondvTape *t) {
    const float mx = ord_value((unsigned)(t->kmax >> 32)), mn = ord_value((unsigned)(t->kmin >> 32));
    const float half = (float)(t->uoutb / 2.0);
    if (mx > 0.0f) {
        const int q = (int)(0xffffffffu - (unsigned)(t->kmax & 0xffffffffu));
        ub[IX(g, g.im, 1 + q % g.jm, 1 + q / g.jm)] += half;
    }
    if (mn < 0.0f) {
        const int q = (int)(unsigned)(t->kmin & 0xffffffffu);
        ub[IX(g, g.im, 1 + q % g.jm, 1 + q / g.jm)] += half;
    }
}

// The n == 1 broadcast x(i,j,k) = x(1,j,k), i = 2..im (when n == 1), then
// the inflow u(0:1,j,k) = wp(j,k), v = w = 0 there: wp's adjoint takes u's
// (accumulated into wpb, FP64), and the inflow planes' adjoints are zero.
__global__ void k_adjb_inflow(Geo g, float *ub, float *vb, float *wb, int n, double *wpb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.jm * g.km) return;
    const int j = 1 + q % g.jm, k = 1 + q / g.jm;
    float *arr[3] = {ub, vb, wb};
    if (n == 1)
        for (int a = 0; a < 3; ++a) {
            float s = arr[a][IX(g, 1, j, k)];
            for (int i = 2; i <= g.im; ++i) {
                s += arr[a][IX(g, i, j, k)];
                arr[a][IX(g, i, j, k)] = 0.0f;
            }
            arr[a][IX(g, 1, j, k)] = s;
        }
    wpb[q] += (double)ub[IX(g, 0, j, k)] + (double)ub[IX(g, 1, j, k)];
    for (int a = 0; a < 3; ++a) {
        arr[a][IX(g, 0, j, k)] = 0.0f;
        arr[a][IX(g, 1, j, k)] = 0.0f;
    }
}

// ---- config-3 objective pieces ----------------------------------------------
// Resolved TKE of a box of cells with the cell-centred velocities of
// anime.f95:45-47: mean of 0.5 (uc^2 + vc^2 + wc^2), uc = 0.5 (u(i-1) + u(i))
// and alike; its sum goes to *sum (FP64).
struct TkeBox {
    int i0, i1, j0, j1, k0, k1;
    __host__ __device__ __forceinline__ int n() const { return (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1); }
};
inline long long b_count(const TkeBox &b) { return b.n(); }
__global__ void __launch_bounds__(256) k_tke_sum(Geo g, const float *u, const float *v, const float *w, TkeBox b,
                                                 double *sum) {
    const int n = b.n(), ni = b.i1 - b.i0 + 1, nj = b.j1 - b.j0 + 1;
    double acc = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int i = b.i0 + q % ni, r = q / ni;
        const int j = b.j0 + r % nj, k = b.k0 + r / nj;
        const double uc = 0.5 * ((double)u[IX(g, i - 1, j, k)] + (double)u[IX(g, i, j, k)]);
        const double vc = 0.5 * ((double)v[IX(g, i, j - 1, k)] + (double)v[IX(g, i, j, k)]);
        const double wc = 0.5 * ((double)w[IX(g, i, j, k - 1)] + (double)w[IX(g, i, j, k)]);
        acc += 0.5 * (uc * uc + vc * vc + wc * wc);
    }
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}
// bar += scale * d(TKE mean)/d(u, v, w): each centred value c sends
// scale / ncells * 0.5 c to both of its points.
__global__ void __launch_bounds__(256) k_tke_seed(Geo g, const float *u, const float *v, const float *w, TkeBox b,
                                                  double scale, float *ubar, float *vbar, float *wbar) {
    const int n = b.n(), ni = b.i1 - b.i0 + 1, nj = b.j1 - b.j0 + 1;
    const double s = scale / n * 0.5;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int i = b.i0 + q % ni, r = q / ni;
        const int j = b.j0 + r % nj, k = b.k0 + r / nj;
        const float gu = (float)(s * 0.5 * ((double)u[IX(g, i - 1, j, k)] + (double)u[IX(g, i, j, k)]));
        const float gv = (float)(s * 0.5 * ((double)v[IX(g, i, j - 1, k)] + (double)v[IX(g, i, j, k)]));
        const float gw = (float)(s * 0.5 * ((double)w[IX(g, i, j, k - 1)] + (double)w[IX(g, i, j, k)]));
        aadd(ubar, g, i - 1, j, k, gu);
        aadd(ubar, g, i, j, k, gu);
        aadd(vbar, g, i, j - 1, k, gv);
        aadd(vbar, g, i, j, k, gv);
        aadd(wbar, g, i, j, k - 1, gw);
        aadd(wbar, g, i, j, k, gw);
    }
}

// Drag-scale gradient: with f += s(i,j) fx (and g, h alike) in feedbf,
// s's adjoint gains sum over k of fx fb + fy gb + fz hb, fx recomputed from
// the step's input usum, vsum, wsum and the velocities after bondv1
// (feedbf.f95:38-67).  One thread per column (i, j), FP64.
__global__ void __launch_bounds__(256) k_adj_drag(Geo g, Fields in, const float *u, const float *v, const float *w,
                                                  const float *fb, const float *gb, const float *hb, double *dragb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.im * g.jm) return;
    const int i = 1 + q % g.im, j = 1 + q / g.im;
    double acc = 0.0;
    for (int k = 1; k <= g.km; ++k) {
        const int c = IX(g, i, j, k);
        const float bm = in.bmask[c], cm = in.cmask[c], dm = in.dmask[c];
        const float us = (in.usum[c] + u[c]) * bm, vs = (in.vsum[c] + v[c]) * cm, ws = (in.wsum[c] + w[c]) * dm;
        const float fx = g.alpha * us * g.dt + g.beta * u[c] * bm;
        const float fy = g.alpha * vs * g.dt + g.beta * v[c] * cm;
        const float fz = g.alpha * ws * g.dt + g.beta * w[c] * dm;
        acc += (double)fx * fb[c] + (double)fy * gb[c] + (double)fz * hb[c];
    }
    dragb[q] += acc;
}

// cn1 = 1/((cnA + cnB) + cnC) (init.f95:87-93) into a box, for the
// transposed sweeps of press.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_cn1(Geo g, float *cn1) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    cn1[IX(g, i, j, k)] = 1.0f / (g.cnA[i] + g.cnB[j] + g.cnC[k]);
}

}  // namespace
}  // namespace les
