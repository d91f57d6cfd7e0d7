// les_dd.cuh -- kernels of the x-decomposed time step (les_dd.inc).
//
// A rank of an x-decomposed domain holds a slab of columns: its own columns
// and up to H halo columns on each side that belong to its neighbours.  The
// halo columns travel as packed blocks (k_dd_pack / k_dd_unpack, the W and E
// parts of the reference's ring-buffer halo, halo_exchange.cl:3-291, here H
// columns wide and every row and plane of the box), and the global sums
// travel as the 32-bit limbs of their exact Q63.64 totals (k_dd_limbs /
// k_dd_unlimbs), whose integer sum over the ranks is the single-domain total.
#pragma once
#include "les_dev.cuh"
#include "les_fix.h"
#include "les_press.cuh"

namespace les {

constexpr int kDDMaxFields = 16;
constexpr int kDDLimbs = 6;  // 4 limbs of the total, the bad flag, spare

struct DDFields {
    float *f[kDDMaxFields];
    int n;
    int pidx;           // index of p in f (-1: none): p is the second buffer palt when sc->pbuf
    float *palt;
    const Scal *sc;
};

namespace {

// buf[((f * rows) + row) * w + c] = field f at column i0 + c of box row
// `row` = (j + 1) + sj * (k + 1), every j in -1..jm+2 and k in -1..km+2.
__global__ void __launch_bounds__(256) k_dd_pack(Geo g, DDFields fs, int i0, int w, float *__restrict__ buf) {
    const long long rows = (long long)g.sj * g.sk, per = rows * w, n = per * fs.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per);
        const long long r = t - f * per;
        const long long row = r / w;
        const int c = (int)(r - row * w);
        const int j = (int)(row % g.sj) - 1, k = (int)(row / g.sj) - 1;
        const float *src = (f == fs.pidx && fs.sc->pbuf) ? fs.palt : fs.f[f];
        buf[t] = src[IX(g, i0 + c, j, k)];
    }
}

__global__ void __launch_bounds__(256) k_dd_unpack(Geo g, DDFields fs, int i0, int w,
                                                   const float *__restrict__ buf) {
    const long long rows = (long long)g.sj * g.sk, per = rows * w, n = per * fs.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per);
        const long long r = t - f * per;
        const long long row = r / w;
        const int c = (int)(r - row * w);
        const int j = (int)(row % g.sj) - 1, k = (int)(row / g.sj) - 1;
        float *dst = (f == fs.pidx && fs.sc->pbuf) ? fs.palt : fs.f[f];
        dst[IX(g, i0 + c, j, k)] = buf[t];
    }
}

// The total of n partial sums part[b * stride] as limbs: out[0..2] the low
// three 32-bit limbs (0..2^32-1), out[3] the top limb (signed), out[4] the
// bad flag.  Summing the limbs of several totals as 64-bit integers is exact
// for up to 2^31 ranks, and the sums fold back into 128 bits (dd_total).
__global__ void __launch_bounds__(1024) k_dd_limbs(const FixPart *part, int n, int stride, long long *out) {
    i128 tot;
    int bad;
    final_fix_strided(part, n, stride, 0, tot, bad);
    if (threadIdx.x == 0) {
        const unsigned __int128 u = (unsigned __int128)tot;
        out[0] = (long long)(unsigned long long)(u & 0xffffffffu);
        out[1] = (long long)(unsigned long long)((u >> 32) & 0xffffffffu);
        out[2] = (long long)(unsigned long long)((u >> 64) & 0xffffffffu);
        out[3] = (long long)(tot >> 96);
        out[4] = bad;
        out[5] = 0;
    }
}

__device__ __forceinline__ i128 dd_total(const long long *in) {
    const unsigned __int128 u = (unsigned __int128)(i128)in[0] + ((unsigned __int128)(i128)in[1] << 32) +
                                ((unsigned __int128)(i128)in[2] << 64) + ((unsigned __int128)(i128)in[3] << 96);
    return (i128)u;
}

__global__ void k_dd_unlimbs(const long long *in, FixPart *part) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    part[0] = fix_to_part(dd_total(in), in[4] != 0);
}

// The stop test of a one-iteration SOR pass (tb_finish_pass with nit = 1)
// on the all-rank residual: the pass wrote the other p buffer, which
// becomes current; a pass after the stop did nothing.
__global__ void k_dd_sor_finish(const long long *in, float pjuge, Scal *s) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || s->converged) return;
    const float sor = (float)fix_finish(dd_total(in), in[4] != 0);
    s->sor = sor;
    s->sor_iters += 1;
    if (sor < pjuge) s->converged = 1;
    s->pbuf ^= 1;
}

// The limbs of every rank of one process on one device: their sums
// (64-bit integers, as an all-reduce forms them) written back to each.
constexpr int kDDMaxLocal = 64;
struct DDLocal {
    long long *s[kDDMaxLocal];
    int n;
};
__global__ void k_dd_local_sum(DDLocal r) {
    const int t = threadIdx.x;
    if (blockIdx.x != 0 || t >= kDDLimbs) return;
    long long v = 0;
    for (int q = 0; q < r.n; ++q) v += r.s[q][t];
    for (int q = 0; q < r.n; ++q) r.s[q][t] = v;
}

}  // namespace
}  // namespace les
