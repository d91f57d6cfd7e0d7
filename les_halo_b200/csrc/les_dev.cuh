// les_dev.cuh -- device layout, metric tables and the vel2 face quantities.
//
// HBM layout: every 3-D field lives in one padded "box" indexed with the
// reference's own (i,j,k) numbering, -1 <= i <= ip+2, -1 <= j <= jp+2,
// -1 <= k <= kp+2, i fastest:
//     idx(i,j,k) = (i + ox) + si * ((j + 1) + sj * (k + 1)),  ox = 31,
// so i = 1 starts a 128-byte line and si (row pitch) is a multiple of 32
// floats.  All fields share the box, so one index serves every stencil.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "les_fix.h"

namespace les {

constexpr int kOX = 31;

struct Geo {
    int im, jm, km;
    int ox, si, sj, sk;
    // columns olo..ohi enter the global sums (rhsav, SOR residual, pav):
    // 1..im, except on a rank of an x-decomposed domain, whose halo columns
    // belong to its neighbours
    int olo, ohi;
    // 1-D tables; each pointer is pre-offset so t[i] is the Fortran t(i).
    const float *dx1, *dy1, *dzn, *dzs, *dxs, *dys;
    const float *cn2l, *cn2s, *cn3l, *cn3s, *cn4l, *cn4s;
    const float *cnA, *cnB, *cnC;  // cn1 = 1/((cnA(i)+cnB(j))+cnC(k)), init.f95:87-93
    const float *smc;              // (cs0*delx1(k))**2, les.f95:128,148
    const float *wind;             // inflow u(0:1,j,k): wind[(j-1) + jm*(k-1)]
    // Exact reciprocals of the x/y divisors that are powers of two, else 0:
    // rdx1(i)=1/dx1(i), rsx(i)=1/(dx1(i)+dx1(i+1)), rdy1, rsy alike.  For a
    // power-of-two divisor d, a*(1/d) and a/d are the correctly rounded
    // value of the same real number, so they are bit-identical.
    const float *rdx1, *rsx, *rdy1, *rsy;
    // RN(1/b) for the k divisors b = dzn(k), dzs(k), dzn(k)+dzn(k+1) (kdiv),
    // 0 where kdiv must divide
    const float *rdzn, *rdzs, *rdzn2;
    float dt, ro, vn, alpha, beta, omega;
    // per-column scale s(i,j) of the IBM force, f += s*fx in feedbf
    // (drag[(i-1) + im*(j-1)]); NULL is the reference's s = 1
    const float *drag;
};

// a/d with d's exact reciprocal r when d is a power of two (r != 0).
__device__ __forceinline__ float fdiv(float a, float d, float r) { return r != 0.0f ? a * r : a / d; }

// a/b given y = RN(1/b): Markstein's correction (P. Markstein, IBM J. Res.
// Dev. 34(1), 1990): q0 = RN(a*y), r = a - b*q0 exactly (one fma),
// q = RN(q0 + r*y) is the correctly rounded a/b.  Used while q0 lies in
// [2^-60, 2^60]; zero, tiny, huge and non-finite quotients (and y = 0, set for
// divisors outside [2^-30, 2^30]) take the IEEE division.  Checked bit for bit
// against IEEE division for every float a on 7564 divisors (stretched-grid
// spacings, their sums, random values): no difference.
__device__ __forceinline__ float kdiv(float a, float b, float y) {
    const float q0 = a * y;
    const float m = fabsf(q0);
    if (!(m >= 0x1p-60f && m <= 0x1p60f)) return a / b;
    const float r = __fmaf_rn(-q0, b, a);
    return __fmaf_rn(r, y, q0);
}

// How the face-value and cell formulas divide.  xd: by an x/y spacing with
// its power-of-two reciprocal r (or 0); zn/zs/zn2: by dzn(k), dzs(k),
// dzn(k)+dzn(k+1).  DivIEEE divides as written; DivPlane (the tile engine)
// holds the divisors and reciprocals of planes kc-1..kc+1 in registers and
// uses kdiv, and with P2 (every x/y spacing a power of two) multiplies by r.
// All forms give the IEEE quotient's bits.
struct DivIEEE {
    __device__ __forceinline__ float xd(float a, float d, float r) const { return fdiv(a, d, r); }
    __device__ __forceinline__ float zn(const Geo &g, float a, int k) const { return a / g.dzn[k]; }
    __device__ __forceinline__ float zs(const Geo &g, float a, int k) const { return a / g.dzs[k]; }
    __device__ __forceinline__ float zn2(const Geo &g, float a, int k) const { return a / (g.dzn[k] + g.dzn[k + 1]); }
};
template <bool P2>
struct DivPlane {
    float bn[3], yn[3], bs[3], ys[3], bn2[3], yn2[3];  // planes kc-1, kc, kc+1
    int kc;
    __device__ __forceinline__ DivPlane(const Geo &g, int kc_) : kc(kc_) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int k = kc - 1 + d;
            bn[d] = g.dzn[k];
            yn[d] = g.rdzn[k];
            bs[d] = g.dzs[k];
            ys[d] = g.rdzs[k];
            bn2[d] = g.dzn[k] + g.dzn[k + 1];
            yn2[d] = g.rdzn2[k];
        }
    }
    __device__ __forceinline__ float xd(float a, float d, float r) const { return P2 ? a * r : fdiv(a, d, r); }
    __device__ __forceinline__ float zn(const Geo &, float a, int k) const {
        return kdiv(a, bn[k - kc + 1], yn[k - kc + 1]);
    }
    __device__ __forceinline__ float zs(const Geo &, float a, int k) const {
        return kdiv(a, bs[k - kc + 1], ys[k - kc + 1]);
    }
    __device__ __forceinline__ float zn2(const Geo &, float a, int k) const {
        return kdiv(a, bn2[k - kc + 1], yn2[k - kc + 1]);
    }
};

struct Fields {
    float *u, *v, *w, *p, *usum, *vsum, *wsum, *f, *g, *h, *fold, *gold, *hold, *rhs, *sm;
    float *amask, *bmask, *cmask, *dmask;
};

// Per-step device scalars.
struct Scal {
    unsigned int uout_pos;  // max of positive u(im,j,k) as float bits
    unsigned int uout_neg;  // max of -u(im,j,k) for negative u, float bits
    float uout, rhsav, pav, sor;
    int sor_iters, converged, n;
    unsigned int ticket;  // blocks of the running SOR pass that have finished (0 between launches)
    int pbuf;  // SOR result buffer: 0 = p, 1 = the second p buffer
    int redo;  // iterations to redo after a pass that converged part-way
    float probe[4];
    int exact_sums;  // 1: the rest of this step's SOR passes sum the residual exactly
};

#ifdef LES_CHECKED
// LES_CHECKED builds (liblesb200_checked.so): every box index is checked
// against the allocation; a miss is counted, the first one's (i, j, k) is
// kept, and the access goes to element 0 instead -- no fault and no trap.
// One record per translation unit; les_bounds_violations reads the time
// step's (les_lib.cu).
struct LesOob {
    unsigned long long count;
    int claimed;
    int first[3];
};
static __device__ LesOob g_les_oob;
static __device__ __noinline__ void les_oob_record(int i, int j, int k) {
    atomicAdd(&g_les_oob.count, 1ull);
    if (atomicCAS(&g_les_oob.claimed, 0, 1) == 0) {
        g_les_oob.first[0] = i;
        g_les_oob.first[1] = j;
        g_les_oob.first[2] = k;
    }
}
#endif

__device__ __forceinline__ int IX(const Geo &g, int i, int j, int k) {
    const int off = (i + g.ox) + g.si * ((j + 1) + g.sj * (k + 1));
#ifdef LES_CHECKED
    if (off < 0 || off >= g.si * g.sj * g.sk) {
        les_oob_record(i, j, k);
        return 0;
    }
#endif
    return off;
}

// ---------------------------------------------------------------------------
// vel2.f95:48-123 face quantities, evaluated on the fly from u, v, w.
// *_raw: the vel2 formula at (i,j,k).  *_e: the value the reference's array
// holds at (i,j,k) after vel2 returns: the formula on its computed range, the
// boundary copies of vel2.f95:125-188, and 0 (from zero_arrays,
// ifdata.f95:15-127) everywhere nothing ever writes.
// ---------------------------------------------------------------------------
// u, v, w read straight from the state boxes.
struct UVW : DivIEEE {
    const float *__restrict__ u;
    const float *__restrict__ v;
    const float *__restrict__ w;
    __device__ __forceinline__ float U(const Geo &g, int i, int j, int k) const { return __ldg(&u[IX(g, i, j, k)]); }
    __device__ __forceinline__ float V(const Geo &g, int i, int j, int k) const { return __ldg(&v[IX(g, i, j, k)]); }
    __device__ __forceinline__ float W(const Geo &g, int i, int j, int k) const { return __ldg(&w[IX(g, i, j, k)]); }
};

#define LU(i, j, k) q.U(g, (i), (j), (k))
#define LV(i, j, k) q.V(g, (i), (j), (k))
#define LW(i, j, k) q.W(g, (i), (j), (k))

template <class Q>
__device__ __forceinline__ float nou1_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return (LU(i - 1, j, k) + LU(i, j, k)) / 2.0f;
}
template <class Q>
__device__ __forceinline__ float diu1_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(-LU(i - 1, j, k) + LU(i, j, k), g.dx1[i], g.rdx1[i]);
}
template <class Q>
__device__ __forceinline__ float nou5_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return (LV(i, j - 1, k) + LV(i, j, k)) / 2.0f;
}
template <class Q>
__device__ __forceinline__ float diu5_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(-LV(i, j - 1, k) + LV(i, j, k), g.dy1[j], g.rdy1[j]);
}
template <class Q>
__device__ __forceinline__ float nou9_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return (LW(i, j, k - 1) + LW(i, j, k)) / 2.0f;
}
template <class Q>
__device__ __forceinline__ float diu9_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.zn(g, -LW(i, j, k - 1) + LW(i, j, k), k);
}
template <class Q>
__device__ __forceinline__ float nou2_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(g.dx1[i + 1] * LV(i, j - 1, k) + g.dx1[i] * LV(i + 1, j - 1, k), g.dx1[i] + g.dx1[i + 1], g.rsx[i]);
}
template <class Q>
__device__ __forceinline__ float diu2_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(2.0f * (-LU(i, j - 1, k) + LU(i, j, k)), g.dy1[j - 1] + g.dy1[j], g.rsy[j - 1]);
}
template <class Q>
__device__ __forceinline__ float nou3_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(g.dx1[i + 1] * LW(i, j, k - 1) + g.dx1[i] * LW(i + 1, j, k - 1), g.dx1[i] + g.dx1[i + 1], g.rsx[i]);
}
template <class Q>
__device__ __forceinline__ float diu3_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.zs(g, -LU(i, j, k - 1) + LU(i, j, k), k - 1);
}
template <class Q>
__device__ __forceinline__ float nou4_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(g.dy1[j + 1] * LU(i - 1, j, k) + g.dy1[j] * LU(i - 1, j + 1, k), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
}
template <class Q>
__device__ __forceinline__ float diu4_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(2.0f * (-LV(i - 1, j, k) + LV(i, j, k)), g.dx1[i - 1] + g.dx1[i], g.rsx[i - 1]);
}
template <class Q>
__device__ __forceinline__ float nou6_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(g.dy1[j + 1] * LW(i, j, k - 1) + g.dy1[j] * LW(i, j + 1, k - 1), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
}
template <class Q>
__device__ __forceinline__ float diu6_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.zs(g, -LV(i, j, k - 1) + LV(i, j, k), k - 1);
}
template <class Q>
__device__ __forceinline__ float nou7_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.zn2(g, g.dzn[k + 1] * LU(i - 1, j, k) + g.dzn[k] * LU(i - 1, j, k + 1), k);
}
template <class Q>
__device__ __forceinline__ float diu7_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(2.0f * (-LW(i - 1, j, k) + LW(i, j, k)), g.dx1[i - 1] + g.dx1[i], g.rsx[i - 1]);
}
template <class Q>
__device__ __forceinline__ float nou8_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.zn2(g, g.dzn[k + 1] * LV(i, j - 1, k) + g.dzn[k] * LV(i, j - 1, k + 1), k);
}
template <class Q>
__device__ __forceinline__ float diu8_raw(const Geo &g, const Q &q, int i, int j, int k) {
    return q.xd(2.0f * (-LW(i, j - 1, k) + LW(i, j, k)), g.dy1[j - 1] + g.dy1[j], g.rsy[j - 1]);
}

// j index of the periodic copies X(i,0,k)=X(i,jm,k), X(i,jm+1,k)=X(i,1,k);
// returns 0 when j is outside 0..jm+1.
__device__ __forceinline__ int jper(const Geo &g, int j) {
    return (j >= 1 && j <= g.jm) ? j : (j == 0 ? g.jm : (j == g.jm + 1 ? 1 : 0));
}

// group 1 (vel2.f95:48-63, copy :125-131): range 1..im x 1..jm x 1..km, i=im+1 <- im
template <class Q>
__device__ __forceinline__ float diu1_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j < 1 || j > g.jm || k < 1 || k > g.km || i < 1 || i > g.im + 1) return 0.0f;
    return diu1_raw(g, q, i > g.im ? g.im : i, j, k);
}
template <class Q>
__device__ __forceinline__ float cov1_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j < 1 || j > g.jm || k < 1 || k > g.km || i < 1 || i > g.im + 1) return 0.0f;
    const int ii = i > g.im ? g.im : i;
    return nou1_raw(g, q, ii, j, k) * diu1_raw(g, q, ii, j, k);
}
// group 5 (copies :149-158): j periodic on 1..im x * x 1..km
template <class Q>
__device__ __forceinline__ float diu5_e(const Geo &g, const Q &q, int i, int j, int k) {
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km || jj == 0) return 0.0f;
    return diu5_raw(g, q, i, jj, k);
}
template <class Q>
__device__ __forceinline__ float cov5_e(const Geo &g, const Q &q, int i, int j, int k) {
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km || jj == 0) return 0.0f;
    return nou5_raw(g, q, i, jj, k) * diu5_raw(g, q, i, jj, k);
}
// group 9: 1..im x 1..jm x 1..km, no copies
template <class Q>
__device__ __forceinline__ float diu9_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km) return 0.0f;
    return diu9_raw(g, q, i, j, k);
}
template <class Q>
__device__ __forceinline__ float cov9_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km) return 0.0f;
    return nou9_raw(g, q, i, j, k) * diu9_raw(g, q, i, j, k);
}
// group 2 (:65-73, copies :132-141), diu2 also (im+1,1..jm+1,1..km+1) <- im (:177-182)
template <class Q>
__device__ __forceinline__ float cov2_e(const Geo &g, const Q &q, int i, int j, int k) {
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km || jj == 0) return 0.0f;
    return nou2_raw(g, q, i, jj, k) * diu2_raw(g, q, i, jj, k);
}
template <class Q>
__device__ __forceinline__ float diu2_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i == g.im + 1) {
        if (j < 1 || j > g.jm + 1 || k < 1 || k > g.km + 1) return 0.0f;
        i = g.im;
    }
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km || jj == 0) return 0.0f;
    return diu2_raw(g, q, i, jj, k);
}
// group 3 (:75-83): 1..im x 1..jm x 1..km+1; diu3 (im+1,1..jm+1,1..km+1) <- im
template <class Q>
__device__ __forceinline__ float cov3_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km + 1) return 0.0f;
    return nou3_raw(g, q, i, j, k) * diu3_raw(g, q, i, j, k);
}
template <class Q>
__device__ __forceinline__ float diu3_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i == g.im + 1) {
        if (j < 1 || j > g.jm + 1 || k < 1 || k > g.km + 1) return 0.0f;
        i = g.im;  // diu3(im, jm+1, k) is never computed: stays 0 below
    }
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km + 1) return 0.0f;
    return diu3_raw(g, q, i, j, k);
}
// group 4 (:85-93, copy :142-148): 1..jm x 1..km, i=im+1 <- im; diu4(1..im+1,0,1..km+1) <- jm (:183-188)
template <class Q>
__device__ __forceinline__ float cov4_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j < 1 || j > g.jm || k < 1 || k > g.km || i < 1 || i > g.im + 1) return 0.0f;
    const int ii = i > g.im ? g.im : i;
    return (nou4_raw(g, q, ii, j, k) - 0.0f) * diu4_raw(g, q, ii, j, k);
}
template <class Q>
__device__ __forceinline__ float diu4_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j == 0 && i >= 1 && i <= g.im + 1 && k >= 1 && k <= g.km + 1) j = g.jm;
    if (j < 1 || j > g.jm || k < 1 || k > g.km || i < 1 || i > g.im + 1) return 0.0f;
    return diu4_raw(g, q, i > g.im ? g.im : i, j, k);
}
// group 6 (:95-103): 1..im x 1..jm x 1..km+1; diu6(1..im+1,0,1..km+1) <- jm
template <class Q>
__device__ __forceinline__ float cov6_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km + 1) return 0.0f;
    return nou6_raw(g, q, i, j, k) * diu6_raw(g, q, i, j, k);
}
template <class Q>
__device__ __forceinline__ float diu6_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j == 0 && i >= 1 && i <= g.im + 1 && k >= 1 && k <= g.km + 1) j = g.jm;
    if (i < 1 || i > g.im || j < 1 || j > g.jm || k < 1 || k > g.km + 1) return 0.0f;
    return diu6_raw(g, q, i, j, k);
}
// group 7 (:105-113, copy :159-165): 1..jm x 1..km-1, i=im+1 <- im
template <class Q>
__device__ __forceinline__ float cov7_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j < 1 || j > g.jm || k < 1 || k > g.km - 1 || i < 1 || i > g.im + 1) return 0.0f;
    const int ii = i > g.im ? g.im : i;
    return (nou7_raw(g, q, ii, j, k) - 0.0f) * diu7_raw(g, q, ii, j, k);
}
template <class Q>
__device__ __forceinline__ float diu7_e(const Geo &g, const Q &q, int i, int j, int k) {
    if (j < 1 || j > g.jm || k < 1 || k > g.km - 1 || i < 1 || i > g.im + 1) return 0.0f;
    return diu7_raw(g, q, i > g.im ? g.im : i, j, k);
}
// group 8 (:115-123, copies :166-175): 1..im x 1..km-1, j periodic
template <class Q>
__device__ __forceinline__ float cov8_e(const Geo &g, const Q &q, int i, int j, int k) {
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km - 1 || jj == 0) return 0.0f;
    return nou8_raw(g, q, i, jj, k) * diu8_raw(g, q, i, jj, k);
}
template <class Q>
__device__ __forceinline__ float diu8_e(const Geo &g, const Q &q, int i, int j, int k) {
    const int jj = jper(g, j);
    if (i < 1 || i > g.im || k < 1 || k > g.km - 1 || jj == 0) return 0.0f;
    return diu8_raw(g, q, i, jj, k);
}

// ---------------------------------------------------------------------------
// Exact block sum of fixed-point terms -> one FixPart per block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ i128 shfl_down_i128(i128 v, int off) {
    unsigned long long lo = (unsigned long long)v;
    long long hi = (long long)(v >> 64);
    lo = __shfl_down_sync(0xffffffffu, lo, off);
    hi = __shfl_down_sync(0xffffffffu, hi, off);
    return (i128)(((unsigned __int128)(unsigned long long)hi << 64) | (unsigned __int128)lo);
}

// All threads of the block must call it.  Returns the block total in thread 0.
template <int NT>
__device__ __forceinline__ void block_fix_sum(i128 v, int bad, FixPart *out) {
    __shared__ unsigned long long s_lo[NT / 32];
    __shared__ long long s_hi[NT / 32];
    __shared__ int s_bad[NT / 32];
    for (int off = 16; off >= 1; off >>= 1) {
        v += shfl_down_i128(v, off);
        bad |= __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = t & 31, wid = t >> 5;
    if (lane == 0) {
        s_lo[wid] = (unsigned long long)v;
        s_hi[wid] = (long long)(v >> 64);
        s_bad[wid] = bad;
    }
    __syncthreads();
    if (t == 0) {
        i128 acc = 0;
        int b = 0;
        for (int w = 0; w < NT / 32; ++w) {
            acc += (i128)(((unsigned __int128)(unsigned long long)s_hi[w] << 64) | (unsigned __int128)s_lo[w]);
            b |= s_bad[w];
        }
        *out = fix_to_part(acc, b);
    }
}

}  // namespace les
