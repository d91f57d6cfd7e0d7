// les_mom.cuh -- momentum kernels built on a 2.5-D tile of face quantities.
//
// vel2.f95 materialises 27 face arrays (nou/diu/cov 1..9) that velFG.f95
// and les.f95 then read around every cell.  Here a CTA owns a 32 x 8 tile of
// (i,j) columns plus a one-cell ring, marches k, and evaluates the 18 values
// diu1..9 / cov1..9 of every ring position once per plane into a two-plane
// shared-memory ring (diu7/diu8 of the plane below are kept aside).  The
// cell formulas then read their neighbours from shared memory.  Each value
// equals what the reference's array holds after vel2 (the formula on its
// computed range, the boundary copies of vel2.f95:125-188, zero elsewhere),
// so results are bit-identical to the per-cell kernels of les_step.cuh.
#pragma once
#include "les_step.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

// tile 32 x 8 cells; 352 threads (11 warps): one per ring position of the
// 34 x 10 face-value planes, so a plane fills in one pass; the first 256
// own the tile's cells
constexpr int kMX = 32, kMY = 8, kMNT = 352;
constexpr int kMEX = kMX + 2, kMEY = kMY + 2, kMPOS = kMEX * kMEY;
static_assert(kMNT % 32 == 0 && kMNT >= kMPOS && kMNT >= kMX * kMY, "one thread per ring position");
enum { V_D1 = 0, V_C1 = 9, NV = 18 };

// u, v, w staged in shared memory: a band of (32+4) x (8+4) columns/rows
// around the tile per plane, five plane slots (k-1..k+2 in use, k+3 loading).
// Band row b holds real row jwrap(jb2 + b); a real row j is found by moving
// it by +-jm into the band.  Valid when the band is not taller than jm.
// band: 36 x 12 positions per plane, four plane slots (three read by a fill,
// one arriving)
constexpr int kBW = kMX + 4, kBH = kMY + 4, kBA = kBW * kBH, kBS = 4;
struct UVWBand : DivIEEE {
    const float *base;  // slot s, field f at base + (s*3 + f)*kBA
    int ib2, jb2;       // real (i, j) of band position (0, 0)
    __device__ __forceinline__ int off(const Geo &g, int i, int j, int k) const {
        int r = j - jb2;
        if (r >= kBH) r -= g.jm;
        if (r < 0) r += g.jm;
        return ((k + 1) % kBS) * 3 * kBA + r * kBW + (i - ib2);
    }
    __device__ __forceinline__ float U(const Geo &g, int i, int j, int k) const { return base[off(g, i, j, k)]; }
    __device__ __forceinline__ float V(const Geo &g, int i, int j, int k) const { return base[off(g, i, j, k) + kBA]; }
    __device__ __forceinline__ float W(const Geo &g, int i, int j, int k) const {
        return base[off(g, i, j, k) + 2 * kBA];
    }
};

// The band for an interior tile: every position of the ring and its +-1
// neighbours lies inside the band without moving by jm, and the plane slots
// around the plane being filled (kc) are looked up once.
template <bool P2>
struct UVWBandFast : DivPlane<P2> {
    const float *sl[4];  // slots of planes kc-1 .. kc+2
    int ib2, jb2;
    __device__ __forceinline__ UVWBandFast(const Geo &g, const float *base, int ib2_, int jb2_, int kc_)
        : DivPlane<P2>(g, kc_), ib2(ib2_), jb2(jb2_) {
        const int kc = kc_;
#pragma unroll
        for (int d = 0; d < 4; ++d) sl[d] = base + ((kc + d) % kBS) * 3 * kBA;  // plane kc-1+d
    }
    __device__ __forceinline__ float at(int f, int i, int j, int k) const {
        return sl[k - this->kc + 1][f * kBA + (j - jb2) * kBW + (i - ib2)];
    }
    __device__ __forceinline__ float U(const Geo &, int i, int j, int k) const { return at(0, i, j, k); }
    __device__ __forceinline__ float V(const Geo &, int i, int j, int k) const { return at(1, i, j, k); }
    __device__ __forceinline__ float W(const Geo &, int i, int j, int k) const { return at(2, i, j, k); }
};

__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cp_async4(void *sdst, const void *gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// The band copies of one thread: plane k of u, v, w moves as 3 x 12 rows of
// 18 float pairs (a row is 36 floats starting at an even box offset:
// ib2 + 31 = 32*bx + 30).  Thread t issues pairs t, t+256, t+512 (< 648);
// the source address at k = 0 and the slot offset are fixed for the whole
// march, so a plane costs one pointer step per copy.  Columns past the box
// row end read the next row (still inside the allocation) and are never used.
struct BandCopies {
    static constexpr int kPairs = 3 * kBH * (kBW / 2), kPer = (kPairs + kMNT - 1) / kMNT;
    const float *src[kPer];  // plane-0 source of each copy (nullptr: none)
    int dst[kPer];           // float offset inside a plane slot
    long long pstride;
    __device__ __forceinline__ BandCopies() : pstride(0) {}
    __device__ __forceinline__ BandCopies(const Geo &g, const Fields &F, int ib2, int jb2) {
        constexpr int npair = kBW / 2;
        pstride = (long long)g.si * g.sj;
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const int e = threadIdx.x + r * kMNT;
            if (e < kPairs) {
                const int f = e / (kBH * npair), rem = e % (kBH * npair);
                const int b = rem / npair, pr = rem % npair;
                const int j = ((jb2 + b - 1) % g.jm + g.jm) % g.jm + 1;  // periodic j
                src[r] = (f == 0 ? F.u : (f == 1 ? F.v : F.w)) + IX(g, ib2 + 2 * pr, j, 0);
                dst[r] = f * kBA + b * kBW + 2 * pr;
            } else {
                src[r] = nullptr;
                dst[r] = 0;
            }
        }
    }
    // Issue the copies of plane k (k in -1..kp+2) into its slot.
    __device__ __forceinline__ void load(float *base, int k) const {
        float *slot = base + ((k + 1) % kBS) * 3 * kBA;
#pragma unroll
        for (int r = 0; r < kPer; ++r)
            if (src[r]) cp_async8(slot + dst[r], src[r] + pstride * k);
    }
};

// diu_n and cov_n at (i,j,k) (n = 1..9), as the arrays hold them after vel2.
template <class Q>
__device__ __forceinline__ void vel2_pair(const Geo &g, const Q &q, int n, int i, int j, int k, float &d, float &c) {
    const int im = g.im, jm = g.jm, km = g.km;
    auto in = [](int x, int a, int b) { return x >= a && x <= b; };
    d = 0.0f;
    c = 0.0f;
    switch (n) {
        case 1:
            if (in(j, 1, jm) && in(k, 1, km) && in(i, 1, im + 1)) {
                const int ii = min(i, im);
                d = diu1_raw(g, q, ii, j, k);
                c = nou1_raw(g, q, ii, j, k) * d;
            }
            break;
        case 5: {
            const int jj = jper(g, j);
            if (jj && in(i, 1, im) && in(k, 1, km)) {
                d = diu5_raw(g, q, i, jj, k);
                c = nou5_raw(g, q, i, jj, k) * d;
            }
        } break;
        case 9:
            if (in(i, 1, im) && in(j, 1, jm) && in(k, 1, km)) {
                d = diu9_raw(g, q, i, j, k);
                c = nou9_raw(g, q, i, j, k) * d;
            }
            break;
        case 2: {
            const int jj = jper(g, j);
            if (jj && in(i, 1, im) && in(k, 1, km)) {
                d = diu2_raw(g, q, i, jj, k);
                c = nou2_raw(g, q, i, jj, k) * d;
            } else if (i == im + 1 && in(j, 1, jm + 1) && in(k, 1, km)) {
                d = diu2_raw(g, q, im, jper(g, j), k);  // vel2.f95:177-182
            }
        } break;
        case 3:
            if (in(i, 1, im) && in(j, 1, jm) && in(k, 1, km + 1)) {
                d = diu3_raw(g, q, i, j, k);
                c = nou3_raw(g, q, i, j, k) * d;
            } else if (i == im + 1 && in(j, 1, jm) && in(k, 1, km + 1)) {
                d = diu3_raw(g, q, im, j, k);
            }
            break;
        case 4:
            if (in(j, 1, jm) && in(k, 1, km) && in(i, 1, im + 1)) {
                const int ii = min(i, im);
                d = diu4_raw(g, q, ii, j, k);
                c = (nou4_raw(g, q, ii, j, k) - 0.0f) * d;
            } else if (j == 0 && in(i, 1, im + 1) && in(k, 1, km)) {
                d = diu4_raw(g, q, min(i, im), jm, k);  // vel2.f95:183-188
            }
            break;
        case 6:
            if (in(i, 1, im) && in(j, 1, jm) && in(k, 1, km + 1)) {
                d = diu6_raw(g, q, i, j, k);
                c = nou6_raw(g, q, i, j, k) * d;
            } else if (j == 0 && in(i, 1, im) && in(k, 1, km + 1)) {
                d = diu6_raw(g, q, i, jm, k);
            }
            break;
        case 7:
            if (in(j, 1, jm) && in(k, 1, km - 1) && in(i, 1, im + 1)) {
                const int ii = min(i, im);
                d = diu7_raw(g, q, ii, j, k);
                c = (nou7_raw(g, q, ii, j, k) - 0.0f) * d;
            }
            break;
        default: {  // 8
            const int jj = jper(g, j);
            if (jj && in(i, 1, im) && in(k, 1, km - 1)) {
                d = diu8_raw(g, q, i, jj, k);
                c = nou8_raw(g, q, i, jj, k) * d;
            }
        } break;
    }
}

// vel2_pair for a position with 1 <= i <= im and 1 <= j <= jm: only the k
// ranges of vel2.f95:48-123 remain (kr bit 0: 1..km, 1: 1..km+1, 2: 1..km-1).
template <class Q>
__device__ __forceinline__ void vel2_pair_in(const Geo &g, const Q &q, int n, int i, int j, int k, int kr, float &d,
                                             float &c) {
    d = 0.0f;
    c = 0.0f;
    switch (n) {
        case 1:
            if (kr & 1) {
                d = diu1_raw(g, q, i, j, k);
                c = nou1_raw(g, q, i, j, k) * d;
            }
            break;
        case 2:
            if (kr & 1) {
                d = diu2_raw(g, q, i, j, k);
                c = nou2_raw(g, q, i, j, k) * d;
            }
            break;
        case 3:
            if (kr & 2) {
                d = diu3_raw(g, q, i, j, k);
                c = nou3_raw(g, q, i, j, k) * d;
            }
            break;
        case 4:
            if (kr & 1) {
                d = diu4_raw(g, q, i, j, k);
                c = (nou4_raw(g, q, i, j, k) - 0.0f) * d;
            }
            break;
        case 5:
            if (kr & 1) {
                d = diu5_raw(g, q, i, j, k);
                c = nou5_raw(g, q, i, j, k) * d;
            }
            break;
        case 6:
            if (kr & 2) {
                d = diu6_raw(g, q, i, j, k);
                c = nou6_raw(g, q, i, j, k) * d;
            }
            break;
        case 7:
            if (kr & 4) {
                d = diu7_raw(g, q, i, j, k);
                c = (nou7_raw(g, q, i, j, k) - 0.0f) * d;
            }
            break;
        case 8:
            if (kr & 4) {
                d = diu8_raw(g, q, i, j, k);
                c = nou8_raw(g, q, i, j, k) * d;
            }
            break;
        default:  // 9
            if (kr & 1) {
                d = diu9_raw(g, q, i, j, k);
                c = nou9_raw(g, q, i, j, k) * d;
            }
            break;
    }
}

// Shared-memory view: plane slots cur (k), nxt (k+1) and prv78 (diu7, diu8
// of k-1), for the cell policies of les_step.cuh.
template <bool P2>
struct TileView : DivPlane<P2> {
    const float *cur, *nxt, *prv7, *prv8;
    int ib, jb, kc;  // i, j of ring position 0 and the current plane
    __device__ __forceinline__ TileView(const Geo &g, const float *cur_, const float *nxt_, const float *p7,
                                        const float *p8, int ib_, int jb_, int kc_)
        : DivPlane<P2>(g, kc_), cur(cur_), nxt(nxt_), prv7(p7), prv8(p8), ib(ib_), jb(jb_), kc(kc_) {}
    __device__ __forceinline__ int pos(int i, int j) const { return (j - jb) * kMEX + (i - ib); }
    __device__ __forceinline__ float dv(int n, int i, int j, int k) const {
        const int p = pos(i, j);
        if (k == kc) return cur[(V_D1 + n - 1) * kMPOS + p];
        if (k == kc + 1) return nxt[(V_D1 + n - 1) * kMPOS + p];
        return (n == 7) ? prv7[p] : prv8[p];  // k == kc-1: only diu7, diu8 are read
    }
    __device__ __forceinline__ float cv(int n, int i, int j, int k) const {
        const int p = pos(i, j);
        return (k == kc ? cur : nxt)[(V_C1 + n - 1) * kMPOS + p];
    }
    __device__ __forceinline__ float d1(int i, int j, int k) const { return dv(1, i, j, k); }
    __device__ __forceinline__ float d2(int i, int j, int k) const { return dv(2, i, j, k); }
    __device__ __forceinline__ float d3(int i, int j, int k) const { return dv(3, i, j, k); }
    __device__ __forceinline__ float d4(int i, int j, int k) const { return dv(4, i, j, k); }
    __device__ __forceinline__ float d5(int i, int j, int k) const { return dv(5, i, j, k); }
    __device__ __forceinline__ float d6(int i, int j, int k) const { return dv(6, i, j, k); }
    __device__ __forceinline__ float d7(int i, int j, int k) const { return dv(7, i, j, k); }
    __device__ __forceinline__ float d8(int i, int j, int k) const { return dv(8, i, j, k); }
    __device__ __forceinline__ float d9(int i, int j, int k) const { return dv(9, i, j, k); }
};

// velFG.f95:58-105 for one cell from the tile.
template <class TV>
__device__ __forceinline__ void velfg_tile(const Geo &g, const TV &t, int i, int j, int k, float &fv, float &gv,
                                           float &hv) {
    const float *dx1 = g.dx1, *dy1 = g.dy1, *dzn = g.dzn;
    {
        float covx1 = t.xd(dx1[i + 1] * t.cv(1, i, j, k) + dx1[i] * t.cv(1, i + 1, j, k), dx1[i] + dx1[i + 1], g.rsx[i]);
        float covy1 = (t.cv(2, i, j, k) + t.cv(2, i, j + 1, k)) / 2.0f;
        float covz1 = (t.cv(3, i, j, k) + t.cv(3, i, j, k + 1)) / 2.0f;
        float covc = covx1 + covy1 + covz1;
        float dfu1 = t.xd(2.0f * (-t.d1(i, j, k) + t.d1(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i]) +
                     t.xd(-t.d2(i, j, k) + t.d2(i, j + 1, k), dy1[j], g.rdy1[j]) +
                     t.zn(g, -t.d3(i, j, k) + t.d3(i, j, k + 1), k);
        fv = (-covc + g.vn * dfu1);
    }
    {
        float covx1 = (t.cv(4, i, j, k) + t.cv(4, i + 1, j, k)) / 2.0f;
        float covy1 = t.xd(dy1[j + 1] * t.cv(5, i, j, k) + dy1[j] * t.cv(5, i, j + 1, k), dy1[j] + dy1[j + 1], g.rsy[j]);
        float covz1 = (t.cv(6, i, j, k) + t.cv(6, i, j, k + 1)) / 2.0f;
        float covc = covx1 + covy1 + covz1;
        float dfv1 = t.xd(-t.d4(i, j, k) + t.d4(i + 1, j, k), dx1[i], g.rdx1[i]) +
                     t.xd(2.0f * (-t.d5(i, j, k) + t.d5(i, j + 1, k)), dy1[j] + dy1[j + 1], g.rsy[j]) +
                     t.zn(g, -t.d6(i, j, k) + t.d6(i, j, k + 1), k);
        gv = (-covc + g.vn * dfv1);
    }
    if (k <= g.km - 1) {
        float covx1 = (t.cv(7, i, j, k) + t.cv(7, i + 1, j, k)) / 2.0f;
        float covy1 = (t.cv(8, i, j, k) + t.cv(8, i, j + 1, k)) / 2.0f;
        float covz1 = t.zn2(g, dzn[k + 1] * t.cv(9, i, j, k) + dzn[k] * t.cv(9, i, j, k + 1), k);
        float covc = covx1 + covy1 + covz1;
        float dfw1 = t.xd(-t.d7(i, j, k) + t.d7(i + 1, j, k), dx1[i], g.rdx1[i]) +
                     t.xd(-t.d8(i, j, k) + t.d8(i, j + 1, k), dy1[j], g.rdy1[j]) +
                     t.zs(g, -t.d9(i, j, k) + t.d9(i, j, k + 1), k);
        hv = (-covc + g.vn * dfw1);
    }
}

// Fill plane slot `dst` with the 18 values of plane k over the ring; copy
// the diu7/diu8 the slot held (plane k-2) into prv7/prv8 first if asked.
// INTERIOR: the whole ring lies in 1..im x 1..jm (see vel2_pair_in).
template <bool DIU_ONLY, bool INTERIOR, class Q>
__device__ __forceinline__ void tile_plane(const Geo &g, const Q &q, float *dst, float *prv7, float *prv8, int ib,
                                           int jb, int k, bool save_prev) {
    const int kr = (k >= 1 && k <= g.km ? 1 : 0) | (k >= 1 && k <= g.km + 1 ? 2 : 0) | (k >= 1 && k <= g.km - 1 ? 4 : 0);
    for (int p = threadIdx.x; p < kMPOS; p += kMNT) {
        const int i = ib + p % kMEX, j = jb + p / kMEX;
        if (save_prev) {
            prv7[p] = dst[(V_D1 + 6) * kMPOS + p];
            prv8[p] = dst[(V_D1 + 7) * kMPOS + p];
        }
#pragma unroll
        for (int n = 1; n <= 9; ++n) {
            float d, c;
            if (INTERIOR)
                vel2_pair_in(g, q, n, i, j, k, kr, d, c);
            else
                vel2_pair(g, q, n, i, j, k, d, c);
            dst[(V_D1 + n - 1) * kMPOS + p] = d;
            if (!DIU_ONLY) dst[(V_C1 + n - 1) * kMPOS + p] = c;
        }
    }
}

// shared memory: two face-value planes (18 or 9 values), diu7/diu8 of the
// plane below, and the u,v,w band slots
// (the viscosity kernel adds its sm planes and edge values, kViscArrays
// position arrays)
constexpr int kViscArrays = 12;
__host__ __device__ constexpr size_t mom_smem(bool diu_only) {
    return sizeof(float) *
           (2 * (diu_only ? 9 : NV) * kMPOS + 2 * kMPOS + kBS * 3 * kBA + (diu_only ? kViscArrays * kMPOS : 0));
}

// Shared-memory view of the viscosity edge values around plane k for
// visc_tile, one value per ring position.  With A = the x-weighted sm
// average at (i+1/2, j) and B = the y-weighted one at (i, j+1/2) of a plane
// (les.f95:170-272): exy = y-average of A, fxy = the same weights on A at
// j-1 and j (les.f95's evsy1 of the u equation), exz = z-average of A
// between k and k+1 (exz0: between k-1 and k), eyz = z-average of B.
struct ViscView {
    const float *s0, *s1;  // sm on planes k, k+1
    const float *exy, *fxy, *exz0, *exz1, *eyz;
};

// les.f95:170-274 viscous flux divergence at one cell, the edge values read
// from the tile (same expressions as visc_cell, evaluated once per position).
template <class TV>
__device__ __forceinline__ void visc_tile(const Geo &g, const TV &d, const ViscView &v, int i, int j, int k, float &vfu,
                                          float &vfv, float &vfw) {
    const float *dx1 = g.dx1, *dy1 = g.dy1;
    const int p = d.pos(i, j);
    {  // x-comp, les.f95:170-201
        float evsx2 = v.s0[p + 1];
        float evsx1 = v.s0[p];
        float evsy2 = v.exy[p];
        float evsy1 = v.fxy[p];
        float evsz2 = v.exz1[p];
        float evsz1 = v.exz0[p];
        float visux2 = (evsx2) * 2.0f * d.d1(i + 1, j, k);
        float visux1 = (evsx1) * 2.0f * d.d1(i, j, k);
        float visuy2 = (evsy2) * (d.d2(i, j + 1, k) + d.d4(i + 1, j, k));
        float visuy1 = (evsy1) * (d.d2(i, j, k) + d.d4(i + 1, j - 1, k));
        float visuz2 = (evsz2) * (d.d3(i, j, k + 1) + d.d7(i + 1, j, k));
        float visuz1 = (evsz1) * (d.d3(i, j, k) + d.d7(i + 1, j, k - 1));
        vfu = d.xd(visux2 - visux1, dx1[i], g.rdx1[i]) + d.xd(visuy2 - visuy1, dy1[j], g.rdy1[j]) +
              d.zn(g, visuz2 - visuz1, k);
    }
    {  // y-comp, les.f95:204-235
        float evsy2 = v.s0[p + kMEX];
        float evsy1 = v.s0[p];
        float evsx2 = v.exy[p];
        float evsx1 = v.exy[p - 1];
        float evsz2 = v.exz1[p];
        float evsz1 = v.exz0[p];
        float visvx2 = (evsx2) * (d.d2(i, j + 1, k) + d.d4(i + 1, j, k));
        float visvx1 = (evsx1) * (d.d2(i - 1, j + 1, k) + d.d4(i, j, k));
        float visvy2 = (evsy2) * 2.0f * d.d5(i, j + 1, k);
        float visvy1 = (evsy1) * 2.0f * d.d5(i, j, k);
        float visvz2 = (evsz2) * (d.d6(i, j, k + 1) + d.d8(i, j + 1, k));
        float visvz1 = (evsz1) * (d.d6(i, j, k) + d.d8(i, j + 1, k - 1));
        vfv = d.xd(visvx2 - visvx1, dx1[i], g.rdx1[i]) + d.xd(visvy2 - visvy1, dy1[j], g.rdy1[j]) +
              d.zn(g, visvz2 - visvz1, k);
    }
    {  // z-comp, les.f95:238-272
        float evsz2 = v.s1[p];
        float evsz1 = v.s0[p];
        float evsx2 = v.exz1[p];
        float evsx1 = v.exz1[p - 1];
        float evsy2 = v.eyz[p];
        float evsy1 = v.eyz[p - kMEX];
        float viswx2 = (evsx2) * (d.d3(i, j, k + 1) + d.d7(i + 1, j, k));
        float viswx1 = (evsx1) * (d.d3(i - 1, j, k + 1) + d.d7(i, j, k));
        float viswy2 = (evsy2) * (d.d6(i, j, k + 1) + d.d8(i, j + 1, k));
        float viswy1 = (evsy1) * (d.d6(i, j - 1, k + 1) + d.d8(i, j, k));
        float viswz2 = (evsz2) * 2.0f * d.d9(i, j, k + 1);
        float viswz1 = (evsz1) * 2.0f * d.d9(i, j, k);
        vfw = d.xd(viswx2 - viswx1, dx1[i], g.rdx1[i]) + d.xd(viswy2 - viswy1, dy1[j], g.rdy1[j]) +
              d.zn(g, viswz2 - viswz1, k);
    }
}

// Shared prologue/march of both momentum kernels: stage u,v,w planes, fill
// the face-value ring plane by plane, call `cell` for every tile cell.
// `pre(k)` runs at the top of plane k's iteration: the cell's global inputs
// loaded there arrive while the plane's face values are being filled.
// The x and y tables a tile reads (dx1, rdx1, rsx at i = ib-1 .. ib+kMEX,
// dy1, rdy1, rsy at j = jb-1 .. jb+kMEY), copied into shared memory at the
// start of an interior tile's march; the Geo the march hands on points its
// x/y tables there (same values, read from shared instead of global memory).
constexpr int kTabX = kMEX + 2, kTabY = kMEY + 2;
__device__ __forceinline__ void tile_tables(const Geo &g0, Geo &g, float *tab, int ib, int jb) {
    const float *srcx[3] = {g0.dx1, g0.rdx1, g0.rsx}, *srcy[3] = {g0.dy1, g0.rdy1, g0.rsy};
    for (int t = threadIdx.x; t < 3 * kTabX + 3 * kTabY; t += blockDim.x) {
        if (t < 3 * kTabX)
            tab[t] = srcx[t / kTabX][ib - 1 + t % kTabX];
        else {
            const int u = t - 3 * kTabX;
            tab[t] = srcy[u / kTabY][jb - 1 + u % kTabY];
        }
    }
    g = g0;
    g.dx1 = tab - (ib - 1);
    g.rdx1 = tab + kTabX - (ib - 1);
    g.rsx = tab + 2 * kTabX - (ib - 1);
    g.dy1 = tab + 3 * kTabX - (jb - 1);
    g.rdy1 = tab + 3 * kTabX + kTabY - (jb - 1);
    g.rsy = tab + 3 * kTabX + 2 * kTabY - (jb - 1);
}

template <bool DIU_ONLY, bool BAND, bool INTERIOR, bool P2, class PreFn, class CellFn>
__device__ __forceinline__ void mom_march(const Geo &g0, const Fields &F, PreFn pre, CellFn cell) {
    extern __shared__ float sh[];
    __shared__ float tabs[3 * kTabX + 3 * kTabY];
    constexpr int NVU = DIU_ONLY ? 9 : NV;
    float *const s0 = sh, *const s1 = sh + NVU * kMPOS;  // the two face-value plane slots
    auto slot = [&](int x) { return x ? s1 : s0; };
    float *prv7 = sh + 2 * NVU * kMPOS, *prv8 = prv7 + kMPOS;
    float *band = prv8 + kMPOS;
    const int i0 = 1 + blockIdx.x * kMX, j0 = 1 + blockIdx.y * kMY;
    const int ib = i0 - 1, jb = j0 - 1;
    Geo gl;
    if (BAND && INTERIOR)
        tile_tables(g0, gl, tabs, ib, jb);  // read after the first barrier below
    else
        gl = g0;
    const Geo &g = gl;
    const UVW qg{{}, F.u, F.v, F.w};
    const UVWBand qb{{}, band, i0 - 2, j0 - 2};
    auto fill = [&](float *dst, int k, bool save) {
        if (BAND && INTERIOR)
            tile_plane<DIU_ONLY, true>(g, UVWBandFast<P2>(g, band, i0 - 2, j0 - 2, k), dst, prv7, prv8, ib, jb, k, save);
        else if (BAND)
            tile_plane<DIU_ONLY, false>(g, qb, dst, prv7, prv8, ib, jb, k, save);
        else
            tile_plane<DIU_ONLY, false>(g, qg, dst, prv7, prv8, ib, jb, k, save);
    };
    const BandCopies bc = BAND ? BandCopies(g, F, i0 - 2, j0 - 2) : BandCopies();
    if (BAND) {  // planes -1..1 and 0..2 fill the first two face planes
        for (int k = -1; k <= 2; ++k) bc.load(band, k);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
    }
    // viscosity edge values (DIU_ONLY: the viscosity kernel): sm planes by
    // plane mod 3 (one arriving by cp.async while two are in use), A, B, exz
    // by plane parity, exy, fxy, eyz of the current plane.  Reads at p+-1 and
    // p+-kMEX past a position array's ends land in neighbouring arrays and
    // only feed positions no cell uses.
    float *vS = band + kBS * 3 * kBA, *vA = vS + 3 * kMPOS, *vB = vA + 2 * kMPOS, *vXZ = vB + 2 * kMPOS;
    float *vXY = vXZ + 2 * kMPOS, *vFXY = vXY + kMPOS, *vYZ = vFXY + kMPOS;
    auto sm_slot = [&](int kk) { return vS + (kk % 3) * kMPOS; };
    auto stage_sm = [&](int kk) {  // issue the copies of sm plane kk into its slot
        float *dst = sm_slot(kk);
        for (int p = threadIdx.x; p < kMPOS; p += kMNT)
            cp_async4(dst + p, F.sm + IX(g, ib + p % kMEX, jb + p / kMEX, kk));
    };
    // A and B of plane kk from its staged sm (les.f95:179-185 inner terms)
    auto plane_ab = [&](const DivPlane<P2> &dv, int kk, bool with_b) {
        const float *S = sm_slot(kk);
        float *A = vA + (kk & 1) * kMPOS, *B = vB + (kk & 1) * kMPOS;
        for (int p = threadIdx.x; p < kMPOS; p += kMNT) {
            const int i = ib + p % kMEX, j = jb + p / kMEX;
            A[p] = dv.xd((g.dx1[i + 1] * S[p] + g.dx1[i] * S[p + 1]), g.dx1[i] + g.dx1[i + 1], g.rsx[i]);
            if (with_b)
                B[p] = dv.xd((g.dy1[j + 1] * S[p] + g.dy1[j] * S[p + kMEX]), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
        }
    };
    if (DIU_ONLY) {
        stage_sm(0);
        stage_sm(1);
        stage_sm(2);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        const DivPlane<P2> d0(g, 0), d1(g, 1);
        plane_ab(d0, 0, false);
        plane_ab(d1, 1, true);
        __syncthreads();
        const float *A0 = vA, *A1 = vA + kMPOS;
        for (int p = threadIdx.x; p < kMPOS; p += kMNT)
            vXZ[p] = d0.zn2(g, g.dzn[1] * A0[p] + g.dzn[0] * A1[p], 0);
    }
    fill(s0, 0, false);
    fill(s1, 1, false);
    __syncthreads();
    if (BAND) {  // plane 3 (needed at k = 1) takes the slot of plane -1, free after the fills
        bc.load(band, 3);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
    }
    // In the march, plane k+3 goes into the slot of plane k-1, whose last
    // reader (the fill of plane k at step k-1) finished before the barrier
    // that ends step k-1.
    for (int k = 1; k <= g.km; ++k) {
        pre(k);
        if (BAND) {  // plane k+3 streams in while plane k+1 is filled from k..k+2
            if (k + 3 <= g.km + 2) bc.load(band, k + 3);
            cp_async_commit();
        }
        // slot (k+1)&1 holds plane k-1: keep its diu7/diu8, then plane k+1
        fill(slot((k + 1) & 1), k + 1, true);
        if (DIU_ONLY && k + 2 <= g.km + 1) stage_sm(k + 2);  // waited for with the band copies
        if (DIU_ONLY) cp_async_commit();
        __syncthreads();
        const TileView<P2> t(g, slot(k & 1), slot((k + 1) & 1), prv7, prv8, ib, jb, k);
        ViscView vv{};
        if (DIU_ONLY) {
            // A, B of plane k+1; exz, eyz between k and k+1; exy, fxy of k
            const float *S1 = sm_slot(k + 1);
            const float *A0 = vA + (k & 1) * kMPOS, *B0 = vB + (k & 1) * kMPOS;
            float *A1 = vA + ((k + 1) & 1) * kMPOS, *B1 = vB + ((k + 1) & 1) * kMPOS;
            float *XZ = vXZ + (k & 1) * kMPOS;
            for (int p = threadIdx.x; p < kMPOS; p += kMNT) {
                const int i = ib + p % kMEX, j = jb + p / kMEX;
                const float a1 =
                    t.xd((g.dx1[i + 1] * S1[p] + g.dx1[i] * S1[p + 1]), g.dx1[i] + g.dx1[i + 1], g.rsx[i]);
                const float b1 =
                    t.xd((g.dy1[j + 1] * S1[p] + g.dy1[j] * S1[p + kMEX]), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
                A1[p] = a1;
                B1[p] = b1;
                XZ[p] = t.zn2(g, (g.dzn[k + 1] * (A0[p]) + g.dzn[k] * (a1)), k);
                vYZ[p] = t.zn2(g, (g.dzn[k + 1] * (B0[p]) + g.dzn[k] * (b1)), k);
                vXY[p] = t.xd((g.dy1[j + 1] * (A0[p]) + g.dy1[j] * (A0[p + kMEX])), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
                vFXY[p] = t.xd((g.dy1[j + 1] * (A0[p - kMEX]) + g.dy1[j] * (A0[p])), g.dy1[j] + g.dy1[j + 1], g.rsy[j]);
            }
            __syncthreads();
            vv = ViscView{sm_slot(k), S1, vXY, vFXY, vXZ + ((k + 1) & 1) * kMPOS, XZ, vYZ};
        }
        cell(g, t, k, vv);
        if (BAND || DIU_ONLY) cp_async_wait<0>();
        __syncthreads();
    }
}

// This CTA's tile ring (i0-1 .. i0+32, j0-1 .. j0+8) inside 1..im x 1..jm,
// with the band in use (see UVWBandFast).
template <bool BAND>
__device__ __forceinline__ bool tile_interior_b(const Geo &g) {
    const int ib = blockIdx.x * kMX, jb = blockIdx.y * kMY;  // i0-1, j0-1
    return BAND && ib >= 1 && ib + kMEX - 1 <= g.im && jb >= 1 && jb + kMEY - 1 <= g.jm;
}
#define tile_interior(g) tile_interior_b<BAND>(g)

// velFG + feedbf + sgs viscosity (les.f95:132-152) for a 32 x 8 tile, all k.
template <bool BAND, bool P2>
__global__ void __launch_bounds__(kMNT) k_mom1(Geo g, Fields F) {
    const int i = 1 + blockIdx.x * kMX + threadIdx.x % kMX, j = 1 + blockIdx.y * kMY + threadIdx.x / kMX;
    const bool mine = threadIdx.x < kMX * kMY && i <= g.im && j <= g.jm;
    // the cell's own inputs of plane k (feedbf.f95:38-66, velFG's h), loaded
    // ahead by pre(k); only this thread writes them
    float h0 = 0, u0 = 0, v0 = 0, w0 = 0, us0 = 0, vs0 = 0, ws0 = 0, bm0 = 0, cm0 = 0, dm0 = 0;
    auto pre = [&](int k) {
        if (!mine) return;
        const int c = IX(g, i, j, k);
        h0 = F.h[c];
        u0 = __ldg(&F.u[c]);
        v0 = __ldg(&F.v[c]);
        w0 = __ldg(&F.w[c]);
        us0 = F.usum[c];
        vs0 = F.vsum[c];
        ws0 = F.wsum[c];
        bm0 = __ldg(&F.bmask[c]);
        cm0 = __ldg(&F.cmask[c]);
        dm0 = __ldg(&F.dmask[c]);
    };
    auto cell = [&](const Geo &g, const TileView<P2> &t, int k, const ViscView &) {
        if (!mine) return;
        const int c = IX(g, i, j, k);
        float fv, gv, hv = h0;
        velfg_tile(g, t, i, j, k, fv, gv, hv);
        // feedbf.f95:38-66 (feedbf_cell with the inputs already loaded)
        const float us = (us0 + u0) * bm0;
        const float vs = (vs0 + v0) * cm0;
        const float ws = (ws0 + w0) * dm0;
        F.usum[c] = us;
        F.vsum[c] = vs;
        F.wsum[c] = ws;
        float f1x = g.alpha * us * g.dt, f1y = g.alpha * vs * g.dt, f1z = g.alpha * ws * g.dt;
        float f2x = g.beta * u0 * bm0, f2y = g.beta * v0 * cm0, f2z = g.beta * w0 * dm0;
        if (g.drag) {  // the adjoint's per-column force scale (s = 1: the reference)
            const float s = g.drag[(i - 1) + g.im * (j - 1)];
            F.f[c] = fv + s * (f1x + f2x);
            F.g[c] = gv + s * (f1y + f2y);
            F.h[c] = hv + s * (f1z + f2z);
        } else {
            F.f[c] = fv + (f1x + f2x);
            F.g[c] = gv + (f1y + f2y);
            F.h[c] = hv + (f1z + f2z);
        }
        F.sm[c] = sgs_sm(g, t, i, j, k);
    };
    if (tile_interior(g))
        mom_march<false, BAND, true, P2>(g, F, pre, cell);
    else
        mom_march<false, BAND, false, P2>(g, F, pre, cell);
}

// les.f95:170-274 viscous terms (+ adam.f95:32-46) for a 32 x 8 tile, all k.
// Three CTAs per SM (at most 62 registers, no spills): 1.91 -> 1.72 ms at
// 600 x 600 x 120 (k_mom1 at three was slower, 2.16 -> 2.25 ms).
template <bool ADAM, bool BAND, bool P2>
__global__ void __launch_bounds__(kMNT, 3) k_mom2(Geo g, Fields F) {
    const int i = 1 + blockIdx.x * kMX + threadIdx.x % kMX, j = 1 + blockIdx.y * kMY + threadIdx.x / kMX;
    const bool mine = threadIdx.x < kMX * kMY && i <= g.im && j <= g.jm;
    // the cell's f, g, h (and fold, gold, hold) of plane k, loaded ahead by
    // pre(k); only this thread writes them
    float f0 = 0, g0 = 0, hh0 = 0, fo0 = 0, go0 = 0, ho0 = 0;
    auto pre = [&](int k) {
        if (!mine) return;
        const int c = IX(g, i, j, k);
        f0 = F.f[c];
        g0 = F.g[c];
        hh0 = F.h[c];
        if (ADAM) {
            fo0 = F.fold[c];
            go0 = F.gold[c];
            ho0 = F.hold[c];
        }
    };
    auto cell = [&](const Geo &g, const TileView<P2> &t, int k, const ViscView &vv) {
        if (!mine) return;
        float vfu, vfv, vfw;
        visc_tile(g, t, vv, i, j, k, vfu, vfv, vfw);
        const int c = IX(g, i, j, k);
        const float fv = f0 + vfu, gv = g0 + vfv, hv = hh0 + vfw;
        if (ADAM) {
            F.f[c] = 1.5f * fv - 0.5f * fo0;
            F.g[c] = 1.5f * gv - 0.5f * go0;
            F.h[c] = 1.5f * hv - 0.5f * ho0;
            F.fold[c] = fv;
            F.gold[c] = gv;
            F.hold[c] = hv;
        } else {
            F.f[c] = fv;
            F.g[c] = gv;
            F.h[c] = hv;
        }
    };
    if (tile_interior(g))
        mom_march<true, BAND, true, P2>(g, F, pre, cell);
    else
        mom_march<true, BAND, false, P2>(g, F, pre, cell);
}

}  // namespace
}  // namespace les
