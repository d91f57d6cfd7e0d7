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
        buf[t] = fs.f[f][IX(g, i0 + c, j, k)];
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
        fs.f[f][IX(g, i0 + c, j, k)] = buf[t];
    }
}

// The total of n partial sums as limbs: out[0..2] the low three 32-bit
// limbs (0..2^32-1), out[3] the top limb (signed), out[4] the bad flag.
// Summing the limbs of several totals as 64-bit integers is exact for up to
// 2^31 ranks, and k_dd_unlimbs folds the sums back into 128 bits.
__global__ void __launch_bounds__(1024) k_dd_limbs(const FixPart *part, int n, long long *out) {
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
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

__global__ void k_dd_unlimbs(const long long *in, FixPart *part) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned __int128 u = (unsigned __int128)(i128)in[0] + ((unsigned __int128)(i128)in[1] << 32) +
                                ((unsigned __int128)(i128)in[2] << 64) + ((unsigned __int128)(i128)in[3] << 96);
    part[0] = fix_to_part((i128)u, in[4] != 0);
}

}  // namespace
}  // namespace les
