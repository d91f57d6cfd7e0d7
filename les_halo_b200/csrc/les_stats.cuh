// les_stats.cuh -- device-resident time statistics of aveflow.f95:42-157.
//
// The statistics live in one device buffer, Fortran order, interior only:
// eleven (ip,jp,kp) arrays followed by seven (ip,kp) arrays (AveArray).
// Each element is updated by exactly one thread with the reference's
// expression and, for the column sums, in the reference's j order, so every
// value is bit-identical to the serial loops.
#pragma once

#include "les_dev.cuh"

namespace les {

// Order of the arrays in the statistics buffer (and in les_aveflow_fields).
enum AveArray {
    AV_U, AV_V, AV_W, AV_P, AV_L, AV_UU, AV_VV, AV_WW, AV_SM, AV_SMSM, AV_UWFX,  // (ip,jp,kp)
    AV_SU, AV_SV, AV_SW, AV_SUU, AV_SVV, AV_SWW, AV_UWFXS,                       // (ip,kp)
    AV_NCELL = AV_UWFX + 1,
    AV_NCOL = AV_UWFXS - AV_SU + 1
};

struct AveBuf {
    float *a;         // AV_NCELL arrays of ncell, then AV_NCOL arrays of ncol
    long long ncell;  // ip*jp*kp
    long long ncol;   // ip*kp
    __host__ __device__ __forceinline__ float *cell(int arr) const { return a + arr * ncell; }
    __host__ __device__ __forceinline__ float *col(int arr) const {
        return a + AV_NCELL * ncell + (arr - AV_SU) * ncol;
    }
};

namespace {

// aveflow.f95:72-88 for a step n >= n1: the running sums of u, v, w, p, sm,
// their squares and the uw flux.  first (n == n1): the sums start from 0
// (0.0 + x, as the reference zeroes and then adds); avel and the column
// sums other than uwfxs are zeroed (aveflow.f95:42-70).
__global__ void k_ave_accum(Geo g, Fields F, AveBuf A, int first) {
    const int ip = g.im, jp = g.jm;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > ip) return;
    const long long t = (long long)(i - 1) + (long long)ip * ((j - 1) + (long long)jp * (k - 1));
    if (first && j == 1) {
        const long long tc = (long long)(i - 1) + (long long)ip * (k - 1);
        for (int a = AV_SU; a <= AV_SWW; ++a) A.col(a)[tc] = 0.0f;
    }
    const int c = IX(g, i, j, k), cm = IX(g, i, j, k - 1);
    const float u = F.u[c], v = F.v[c], w = F.w[c], p = F.p[c], sm = F.sm[c];
    const float um = F.u[cm], wm = F.w[cm], wme = F.w[cm + 1];
    auto add = [&](int a, float x) {
        float *q = A.cell(a) + t;
        *q = (first ? 0.0f : *q) + x;
    };
    add(AV_U, u);
    add(AV_V, v);
    add(AV_W, w);
    add(AV_P, p);
    add(AV_UU, u * u);
    add(AV_VV, v * v);
    add(AV_WW, w * w);
    add(AV_SM, sm);
    add(AV_SMSM, sm * sm);
    add(AV_UWFX, 0.5f * (um + u) * 0.5f * (wm + wme));
    if (first) A.cell(AV_L)[t] = 0.0f;
}

// k_ave_accum for four consecutive i per thread (ip a multiple of 4): the
// box rows start on 128-byte boundaries at i = 1 and the dense (ip,jp,kp)
// rows on 16-byte ones, so every access is a 16-byte vector except the
// fifth w(i+4,j,k-1).  Same per-element expressions.
__global__ void k_ave_accum4(Geo g, Fields F, AveBuf A, int first) {
    const int ip = g.im, jp = g.jm;
    const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x) + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > ip) return;
    const long long t = (long long)(i - 1) + (long long)ip * ((j - 1) + (long long)jp * (k - 1));
    if (first && j == 1) {
        const long long tc = (long long)(i - 1) + (long long)ip * (k - 1);
        for (int a = AV_SU; a <= AV_SWW; ++a)
            *reinterpret_cast<float4 *>(A.col(a) + tc) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    const int c = IX(g, i, j, k), cm = IX(g, i, j, k - 1);
    auto ld = [](const float *p) { return *reinterpret_cast<const float4 *>(p); };
    const float4 u4 = ld(F.u + c), v4 = ld(F.v + c), w4 = ld(F.w + c), p4 = ld(F.p + c), s4 = ld(F.sm + c);
    const float4 um4 = ld(F.u + cm), wm4 = ld(F.w + cm);
    const float wm5 = F.w[cm + 4];
    const float u[4] = {u4.x, u4.y, u4.z, u4.w}, v[4] = {v4.x, v4.y, v4.z, v4.w};
    const float w[4] = {w4.x, w4.y, w4.z, w4.w}, p[4] = {p4.x, p4.y, p4.z, p4.w};
    const float sm[4] = {s4.x, s4.y, s4.z, s4.w}, um[4] = {um4.x, um4.y, um4.z, um4.w};
    const float wm[5] = {wm4.x, wm4.y, wm4.z, wm4.w, wm5};
    auto add = [&](int a, const float *x) {
        float4 *q = reinterpret_cast<float4 *>(A.cell(a) + t);
        const float4 o = first ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : *q;
        *q = make_float4(o.x + x[0], o.y + x[1], o.z + x[2], o.w + x[3]);
    };
    float x[4];
    add(AV_U, u);
    add(AV_V, v);
    add(AV_W, w);
    add(AV_P, p);
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = u[e] * u[e];
    add(AV_UU, x);
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = v[e] * v[e];
    add(AV_VV, x);
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = w[e] * w[e];
    add(AV_WW, x);
    add(AV_SM, sm);
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = sm[e] * sm[e];
    add(AV_SMSM, x);
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = 0.5f * (um[e] + u[e]) * 0.5f * (wm[e] + wm[e + 1]);
    add(AV_UWFX, x);
    if (first) *reinterpret_cast<float4 *>(A.cell(AV_L) + t) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// aveflow.f95:92-108: the ten time means (avel included).
__global__ void k_ave_divide(AveBuf A, float cnt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.ncell) return;
    for (int a = AV_U; a <= AV_SMSM; ++a) A.cell(a)[t] = A.cell(a)[t] / cnt;
}

// aveflow.f95:109-116: uwfx minus the product of the means.  aveu(i,j,k-1),
// avew(i,j,k-1) and avew(i+1,j,k-1) are read at their Fortran flattened
// index in the (ip,jp,kp) arrays, so avew(ip+1,j,k-1) is avew(1,j+1,k-1)
// as in the reference; at k = 1 an index before the first element reads 0
// (the reference reads memory outside the arrays there).
__global__ void k_ave_uwfx(AveBuf A, long long plane, float cnt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.ncell) return;
    const float *au = A.cell(AV_U), *aw = A.cell(AV_W);
    const long long tm = t - plane;
    const float aum = tm >= 0 ? au[tm] : 0.0f;
    const float awm = tm >= 0 ? aw[tm] : 0.0f;
    const float awme = tm + 1 >= 0 ? aw[tm + 1] : 0.0f;
    float *x = A.cell(AV_UWFX) + t;
    *x = *x / cnt - 0.5f * (aum + au[t]) * 0.5f * (awm + awme);
}

// aveflow.f95:117-157 for one (i,k) column per thread: the j sums of the
// means (in increasing j, continuing from the column arrays' values), the
// rms of the cells (each cell read for its sum first), the j means and the
// rms of the column means.
__global__ void k_ave_columns(AveBuf A, int ip, int jp, float rjm) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.ncol) return;
    const long long i0 = t % ip, k0 = t / ip;
    float su = A.col(AV_SU)[t], sv = A.col(AV_SV)[t], sw = A.col(AV_SW)[t];
    float suu = A.col(AV_SUU)[t], svv = A.col(AV_SVV)[t], sww = A.col(AV_SWW)[t], sx = A.col(AV_UWFXS)[t];
    float *au = A.cell(AV_U), *av = A.cell(AV_V), *aw = A.cell(AV_W);
    float *auu = A.cell(AV_UU), *avv = A.cell(AV_VV), *aww = A.cell(AV_WW), *ax = A.cell(AV_UWFX);
    for (int j = 0; j < jp; ++j) {
        const long long c = i0 + (long long)ip * (j + (long long)jp * k0);
        const float u = au[c], v = av[c], w = aw[c], uu = auu[c], vv = avv[c], ww = aww[c];
        su = su + u;
        sv = sv + v;
        sw = sw + w;
        suu = suu + uu;
        svv = svv + vv;
        sww = sww + ww;
        sx = sx + ax[c];
        auu[c] = sqrtf(fabsf(uu - u * u));
        avv[c] = sqrtf(fabsf(vv - v * v));
        aww[c] = sqrtf(fabsf(ww - w * w));
    }
    su = su / rjm;
    sv = sv / rjm;
    sw = sw / rjm;
    suu = suu / rjm;
    svv = svv / rjm;
    sww = sww / rjm;
    sx = sx / rjm;
    A.col(AV_SU)[t] = su;
    A.col(AV_SV)[t] = sv;
    A.col(AV_SW)[t] = sw;
    A.col(AV_SUU)[t] = sqrtf(fabsf(suu - su * su));
    A.col(AV_SVV)[t] = sqrtf(fabsf(svv - sv * sv));
    A.col(AV_SWW)[t] = sqrtf(fabsf(sww - sw * sw));
    A.col(AV_UWFXS)[t] = sx;
}

}  // namespace
}  // namespace les
