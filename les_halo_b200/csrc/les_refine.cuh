// les_refine.cuh -- FP64 defect correction of the pressure solve.
//
// The plain press (press.f95:49-146) relaxes, by FP32 red-black SOR,
//     cn2l p_e + cn2s p_w + cn3l p_n + cn3s p_s + cn4l p_u + cn4s p_d - p / cn1 = rhs - rhsav,
// with the neighbours of the boundary cells given by boundp1/boundp2 (i and
// k Neumann: the cell itself; j periodic).  The refined press solves the
// same operator in FP64 with its diagonal the sum of the six coefficients,
//     (A p)(c) = cn2l p_e + cn2s p_w + cn3l p_n + cn3s p_s + cn4l p_u + cn4s p_d - (cn2l+cn2s+cn3l+cn3s+cn4l+cn4s) p,
// which makes A exactly singular with the constants as its null space, as
// the continuous Neumann/periodic problem is.  A e = b then has a solution
// only if b is orthogonal to A's left null vector w = wx(i) wy(j) wz(k)
// (wz(k+1) cn4s(k+1) = wz(k) cn4l(k), likewise in x and y); on a stretched
// grid the reference's rhsav weights (dx1 dy1 dzn) are not w, so b = rhs - mu
// with mu the w-weighted mean of rhs (the reference's rhsav cancels).  The
// FP32 sweeps are kept, then an FP64 outer loop: p64 = p; repeatedly
// r = b - A p64 in FP64, A e = r by the inner solve from e = 0, p64 += e.
// The inner solve is either `inner` FP32 SOR iterations (the same passes) or,
// for uniform x and y spacing, the FP64 spectral solve of les_spectral.cuh.
// Every pointwise expression below has a fixed operand order, the same in
// the oracle's restatement (oracle_refine_tail).
#pragma once

#include "les_press.cuh"

namespace les {

// FP64 scalars of the refined press.
struct Ref64 {
    double rhsav;        // FP64 mean of rhs (press.f95:138, dx1 dy1 dzn weights)
    double bshift;       // mean of rhs with the weights of A's left null vector
    double pav;          // FP64 mean of the refined p
    double bnorm2;       // sum of b^2
    double rel_initial;  // ||b - A p||2 / ||b||2 after the FP32 sweeps
    double rel_final;    // the same after the last correction
    int outer;           // corrections applied
    int stop;            // 1: the tolerance was met, later corrections are skipped
};

namespace {

// Sum over a block of whole warps, returned to thread 0 (fixed order).
__device__ __forceinline__ double2 block_sum_d2(double2 v) {
    __shared__ double2 s_d[32];
    for (int off = 16; off >= 1; off >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, off);
        v.y += __shfl_down_sync(0xffffffffu, v.y, off);
    }
    const int nt = blockDim.x * blockDim.y;
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    if ((t & 31) == 0) s_d[t >> 5] = v;
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (t == 0)
        for (int w = 0; w < nt / 32; ++w) r.x += s_d[w].x, r.y += s_d[w].y;
    return r;
}

// FP64 rhsav from the exact partial sums of k_rhs: the value the plain
// press rounds to FP32 (press.f95:138).
__global__ void __launch_bounds__(1024) k_ref_rhsav(const FixPart *part, int n, double area, Ref64 *R) {
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
    if (threadIdx.x == 0) {
        R->rhsav = fix_finish(tot, bad) / area;
        R->outer = 0;
        R->stop = 0;
    }
}

// Sums of w*rhs and w over the interior (w = wx wy wz, FP64).
__global__ void __launch_bounds__(kRedNT) k_ref_wmean(Geo g, const float *rhs, const double *wx, const double *wy,
                                                       const double *wz, int kchunk, double2 *part) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    double2 acc = make_double2(0.0, 0.0);
    if (i <= g.im && j <= g.jm) {
        const double wxy = wx[i - 1] * wy[j - 1];
        for (int k = k0; k <= k1; ++k) {
            const double w = wxy * wz[k - 1];
            acc.x += w * (double)rhs[IX(g, i, j, k)];
            acc.y += w;
        }
    }
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0)
        part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = v;
}

__global__ void __launch_bounds__(1024) k_ref_wmean_final(const double2 *part, int n, Ref64 *R) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) acc.x += part[t].x, acc.y += part[t].y;
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0) R->bshift = v.x / v.y;
}

// Position of i (1-based) in the even-then-reversed-odd order of a line of
// n (even) values that turns a DCT-II into one real FFT (Makhoul 1980).
__host__ __device__ __forceinline__ int makhoul_pos(int i, int n) {
    const int i0 = i - 1;
    return (i0 & 1) ? n - 1 - (i0 >> 1) : (i0 >> 1);
}

// r = b - A p64 on the interior (FP64) and per-block sums of r^2 and b^2.
// SPEC: r goes to the dense FP64 lines (k, j) of the spectral solve, in
// makhoul_pos order; else r32 = (float) r in the box for the inner sweeps.
// FIRST: p64 is the FP32 SOR result (read from the buffer Scal::pbuf
// names) and is stored.
template <bool FIRST, bool SPEC>
__global__ void __launch_bounds__(kRedNT) k_ref_defect(Geo g, const float *rhs, const float *p0, const float *p1,
                                                        const Scal *sc, double *p64, float *r32, double *rline,
                                                        int kchunk, const Ref64 *R, double2 *part) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    double2 acc = make_double2(0.0, 0.0);
    if (i <= g.im && j <= g.jm && !(R->stop && !FIRST)) {
        // the defect's outputs (rline or r32, and p64 below) are no location
        // the loop reads
        const float *__restrict__ p32 = sc->pbuf ? p1 : p0;
        const double *__restrict__ p64r = p64;
        double *__restrict__ rl = rline;
        float *__restrict__ r32o = r32;
        const int jn = (j == g.jm) ? 1 : j + 1, js = (j == 1) ? g.jm : j - 1;
        const double c2l = g.cn2l[i], c2s = g.cn2s[i], c3l = g.cn3l[j], c3s = g.cn3s[j];
        const double bsh = R->bshift;
        auto P = [&](int ii, int jj, int kk) -> double {
            const int c = IX(g, ii, jj, kk);
            return FIRST ? (double)p32[c] : p64r[c];
        };
        // the k neighbours move through registers from one plane to the next
        double pc = P(i, j, k0);
        double pd = (k0 == 1) ? pc : P(i, j, k0 - 1);
        for (int k = k0; k <= k1; ++k) {
            const int c = IX(g, i, j, k);
            const double pe = (i == g.im) ? pc : P(i + 1, j, k);
            const double pw = (i == 1) ? pc : P(i - 1, j, k);
            const double pn = P(i, jn, k), ps = P(i, js, k);
            const double pu = (k == g.km) ? pc : P(i, j, k + 1);
            const double c4l = g.cn4l[k], c4s = g.cn4s[k];
            const double diag = ((((c2l + c2s) + c3l) + c3s) + c4l) + c4s;
            double s = c2l * pe;
            s = s + c2s * pw;
            s = s + c3l * pn;
            s = s + c3s * ps;
            s = s + c4l * pu;
            s = s + c4s * pd;
            const double ap = s - pc * diag;
            const double b = (double)rhs[c] - bsh;
            const double r = b - ap;
            if (SPEC)
                rl[((size_t)(k - 1) * g.jm + (j - 1)) * g.im + makhoul_pos(i, g.im)] = r;
            else
                r32o[c] = (float)r;
            acc.x += r * r;
            if (FIRST) acc.y += b * b;
            pd = pc;
            pc = pu;
        }
    }
    // FIRST stores p64 only after every read of this block is done: other
    // blocks read p32, never p64, so the order between blocks does not matter
    if (FIRST && i <= g.im && j <= g.jm) {
        const float *p32 = sc->pbuf ? p1 : p0;
        for (int k = k0; k <= k1; ++k) p64[IX(g, i, j, k)] = (double)p32[IX(g, i, j, k)];
    }
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0)
        part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = v;
}

// The residual norm of the last defect (one block, fixed order) and the
// stop test rel <= tol.
__global__ void __launch_bounds__(1024) k_ref_norm(const double2 *part, int n, Ref64 *R, double tol, int first) {
    if (R->stop && !first) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) acc.x += part[t].x, acc.y += part[t].y;
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0) {
        if (first) R->bnorm2 = v.y;
        const double rel = R->bnorm2 > 0.0 ? sqrt(v.x / R->bnorm2) : 0.0;
        if (first) R->rel_initial = rel;
        R->rel_final = rel;
        if (rel <= tol) R->stop = 1;
    }
}

// Scalars of one inner solve (A e = r from e = 0): no rhsav, and nothing
// to do once the outer loop has stopped.
__global__ void k_ref_inner_begin(Scal *s, const Ref64 *R) {
    s->rhsav = 0.0f;
    s->converged = R->stop;
    s->sor_iters = 0;
    s->redo = 0;
    s->pbuf = 0;
    s->exact_sums = 0;
}

// p64 += e on the interior (e from the buffer the inner solve ended in).
__global__ void __launch_bounds__(kRedNT) k_ref_correct(Geo g, double *p64, const float *e0, const float *e1,
                                                         const Scal *s2, Ref64 *R) {
    if (R->stop) return;
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0)
        R->outer += 1;
    if (i > g.im || j > g.jm) return;
    const float *e = s2->pbuf ? e1 : e0;
    const int c = IX(g, i, j, k);
    p64[c] = p64[c] + (double)e[c];
}

// press.f95:123-133 in FP64: sums of p64 * w and w, w = dx1 * dy1 * dzn.
__global__ void __launch_bounds__(kRedNT) k_ref_pav_reduce(Geo g, const double *p64, int kchunk, double2 *part) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    double2 acc = make_double2(0.0, 0.0);
    if (i <= g.im && j <= g.jm) {
        for (int k = k0; k <= k1; ++k) {
            const double w = (double)g.dx1[i] * (double)g.dy1[j] * (double)g.dzn[k];
            acc.x += p64[IX(g, i, j, k)] * w;
            acc.y += w;
        }
    }
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0)
        part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = v;
}

__global__ void __launch_bounds__(1024) k_ref_pav_final(const double2 *part, int n, Ref64 *R, Scal *s) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) acc.x += part[t].x, acc.y += part[t].y;
    const double2 v = block_sum_d2(acc);
    if (threadIdx.x == 0) {
        R->pav = v.x / v.y;
        s->pav = (float)R->pav;
    }
}

// p = (float)(p64 - pav) on the interior and its boundp1/boundp2 copies
// (the ghost writes of k_pav_adjust).
__global__ void __launch_bounds__(kRedNT) k_ref_finish(Geo g, float *p, const double *p64, const Ref64 *R) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const float val = (float)(p64[IX(g, i, j, k)] - R->pav);
    const int ie = (i == 1) ? 0 : (i == g.im ? g.im + 1 : -9);
    const int je = (j == g.jm) ? 0 : (j == 1 ? g.jm + 1 : -9);
    const int ke = (k == 1) ? 0 : (k == g.km ? g.km + 1 : -9);
    auto put = [&](int kk) {
        p[IX(g, i, j, kk)] = val;
        if (ie != -9) p[IX(g, ie, j, kk)] = val;
        if (je != -9) {
            p[IX(g, i, je, kk)] = val;
            if (ie != -9) p[IX(g, ie, je, kk)] = val;
        }
    };
    put(k);
    if (ke != -9) put(ke);
}

}  // namespace
}  // namespace les
