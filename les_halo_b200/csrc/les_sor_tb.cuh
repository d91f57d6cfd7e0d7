// les_sor_tb.cuh -- red-black SOR with several iterations per pass over HBM.
//
// press.f95:87-115 updates p in place, colour nrd=0 then nrd=1, refreshing
// the i/j ghosts after each colour (boundp1) and the k ghosts after each
// iteration (boundp2).  Followed through, every ghost a sweep reads then
// holds a current interior value: the i and k Neumann ghosts equal the
// updated cell's own value, and for even jm the periodic j ghost equals its
// partner (of the other colour) as last updated.  The ghosts are overwritten
// by the final boundp1/boundp2 of press.f95:207-209 before anything else
// reads them.  So for even jm the SOR is a plain red-black Gauss-Seidel on
// the interior with i/k mirror and j periodic neighbours, and a CTA can run
// several half-sweeps per pass (a skewed wavefront along k, temporal
// blocking):
//   - a CTA owns a (64 - 4T) x ty tile of (i,j) columns, a chunk of k, and
//     a ring of R = 2T cells (and planes) around them; half-sweep s updates
//     the region shrunk by s+1 on every side, so after 2T half-sweeps the
//     tile holds exact values;
//   - planes march upward: at step tau half-sweep s works on plane tau-s,
//     in order s = 0,1,.., so each plane sees its neighbours at the right
//     level;
//   - a warp owns whole region rows (64 columns), lane l the column pair
//     2l, 2l+1, whose values on the last 2T+2 planes stay in registers: the
//     k neighbours and the own x neighbour come from registers, the other x
//     neighbour from the adjacent lane (one shuffle), the j neighbours from
//     a shared copy of the plane (parity-split rows: x -> (x&1)*32 + x/2, so
//     a colour's cells and their j neighbours are bank-conflict free);
//   - within a step every half-sweep works on its own plane and reads only
//     the other colour, written in earlier steps: one barrier per step;
//   - planes are staged with cp.async kTbDepth steps ahead of their use;
//   - p is read from one buffer and written to the other (nothing a
//     neighbouring CTA reads is overwritten);
//   - reltmp^2 of the tile cells is summed per iteration (les_fix.h) and the
//     last block to finish applies the stop test of press.f95:114.
// A pass that converges part-way (sor < pjuge before its last iteration) is
// redone from its input buffer with exactly the iterations the reference
// executes.
#pragma once
#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

constexpr int kTbRW = 64;     // region row: 64 columns, lane l owns 2l and 2l+1
constexpr int kTbTMax = 3;    // iterations per pass
constexpr int kTbDepth = 2;   // planes requested ahead of the one a step needs
constexpr int kTbMaxRH = 64;  // region rows
constexpr int kTbMaxChunks = 8;

__host__ __device__ constexpr int tb_ring(int T) { return 2 * T; }
// tile columns: the 64-column region minus a ring on each side
__host__ __device__ constexpr int tb_tx(int T) { return kTbRW - 2 * tb_ring(T); }
// shared plane slots (p and rhs each): 2T planes in work, the incoming one,
// kTbDepth in flight and one of slack so a request never hits a plane a
// slower warp may still read
__host__ __device__ constexpr int tb_ns(int T) { return 2 * T + 2 + kTbDepth; }
__host__ __device__ inline int tb_rh(int T, int ty) { return ty + 2 * tb_ring(T); }
__host__ __device__ inline int tb_warps(int T, int ty, int rpw) { return (tb_rh(T, ty) + rpw - 1) / rpw; }
__host__ __device__ inline size_t tb_smem(int T, int ty) {
    return sizeof(float) * 2 * (size_t)kTbRW * tb_rh(T, ty) * tb_ns(T);
}
__host__ __device__ inline bool tb_fits(int T, int ty, int rpw) {
    return T >= 1 && T <= kTbTMax && ty >= 1 && (rpw == 1 || rpw == 2) && tb_rh(T, ty) <= kTbMaxRH &&
           tb_warps(T, ty, rpw) <= (rpw == 1 ? 32 : 16);  // the kernels' launch bounds
}

struct TbArgs {
    float *pb0, *pb1;         // the two p buffers (Scal::pbuf says which is current)
    const float *rhs;         // raw rhs (rhsav not yet subtracted)
    const float *cn1k;        // cn1 per k when it depends on k only
    int ty, kc, niter, mode;  // tile rows, planes per k chunk, iterations, 0 pass / 1 redo
    float pjuge;              // stop threshold (press.f95:107)
    FixPart *part;            // kTbTMax partial sums per block
    Scal *sc;
};

// Exact Q63.64 term (les_fix.h) of a non-negative float below 2^62: the
// integer part and the fraction scaled by 2^64, both exact in FP64; a term
// below 1 needs only the fraction.
__device__ __forceinline__ void fix_add_nonneg(float x, unsigned long long &hi, unsigned long long &lo, int &bad) {
    unsigned long long fr, ip;
    if (x < 1.0f) {
        fr = __double2ull_rz((double)x * 18446744073709551616.0);
        ip = 0ull;
    } else if (x < 4.611686018427388e18f) {
        const double d = (double)x;
        const double f = floor(d);
        fr = __double2ull_rz((d - f) * 18446744073709551616.0);
        ip = (unsigned long long)f;
    } else {  // NaN, inf or >= 2^62
        bad = 1;
        return;
    }
    const unsigned long long o = lo;
    lo += fr;
    hi += ip + (lo < o ? 1ull : 0ull);
}

// block_fix_sum for any block of whole warps (up to 1024 threads).
__device__ __forceinline__ void block_fix_sum_any(i128 v, int bad, FixPart *out) {
    __shared__ unsigned long long s_lo[32];
    __shared__ long long s_hi[32];
    __shared__ int s_bad[32];
    for (int off = 16; off >= 1; off >>= 1) {
        v += shfl_down_i128(v, off);
        bad |= __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_lo[wid] = (unsigned long long)v;
        s_hi[wid] = (long long)(v >> 64);
        s_bad[wid] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        i128 acc = 0;
        int b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            acc += (i128)(((unsigned __int128)(unsigned long long)s_hi[w] << 64) | (unsigned __int128)s_lo[w]);
            b |= s_bad[w];
        }
        *out = fix_to_part(acc, b);
    }
}

__device__ __forceinline__ void tb_cp_async4(float *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void tb_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void tb_cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stop test of press.f95:114 for each iteration of the pass, in order (run
// by the last block of a pass).  A pass that stopped before its last
// iteration is marked for a redo of that many iterations; otherwise the
// output buffer becomes current.
__device__ void tb_finish_pass(const FixPart *part, int nblocks, int nit, float pjuge, Scal *s) {
    __shared__ int stop;
    for (int t = 0; t < nit; ++t) {
        i128 tot;
        int bad;
        final_fix_strided(part, nblocks, kTbTMax, t, tot, bad);
        if (threadIdx.x == 0) {
            const float sor = (float)fix_finish(tot, bad);
            s->sor = sor;
            s->sor_iters += 1;
            stop = 0;
            if (sor < pjuge) {
                s->converged = 1;
                if (t < nit - 1) s->redo = t + 1;
                stop = 1;
            }
        }
        __syncthreads();
        if (stop) break;
    }
    if (threadIdx.x == 0 && s->redo == 0) s->pbuf ^= 1;
}

// One pass of niter <= T iterations (mode 0), or the redo of scal->redo
// iterations after a pass that converged part-way (mode 1).
// CN1K: cn1 depends on k only (uniform dx and dy), read from cn1k[k].
// RPW: region rows per warp (blockDim.x = 32 * tb_warps(T, ty, RPW); two
// rows per warp trade warps for registers, so at most 512 threads).
template <int T, bool CN1K, int RPW>
__global__ void __launch_bounds__(RPW == 1 ? 1024 : 512) k_sor_tb(Geo g, TbArgs a) {
    extern __shared__ float smem[];
    Scal *sc = a.sc;
    const bool redo = (a.mode == 1);
    if (!redo && sc->converged) return;
    const int nit = redo ? sc->redo : a.niter;
    if (nit <= 0) return;
    constexpr int R = tb_ring(T), TX = tb_tx(T), NS = tb_ns(T), D = kTbDepth, W = 2 * T + 2;
    const int nhs = 2 * nit;
    const int ty = a.ty, RH = ty + 2 * R, RA = kTbRW * RH;
    float *P = smem;          // NS plane slots of p
    float *Bs = P + NS * RA;  // NS plane slots of rhs
    const float *pin = sc->pbuf ? a.pb1 : a.pb0;
    float *pout = sc->pbuf ? a.pb0 : a.pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ir0 = 1 + blockIdx.x * TX - R, jr0 = 1 + blockIdx.y * ty - R;
    const int k0 = 1 + blockIdx.z * a.kc, k1 = min(km, k0 + a.kc - 1);
    const int kb = max(1, k0 - R), ke = min(km, k1 + R);
    const long long pstride = (long long)g.si * g.sj;
    const int dA = (lane & 1) * 32 + (lane >> 1);  // parity-split slot of column `lane`

    // owned rows: region row, box offset of (ir0, j, k=0), j coefficients
    int ry[RPW], roff[RPW];
    bool rok[RPW];
    float c3l[RPW], c3s[RPW], cB[RPW];
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
        ry[r] = warp + nw * r;
        rok[r] = ry[r] < RH;
        const int jw = ((jr0 + ry[r] - 1) % jm + jm) % jm + 1;  // periodic j (jm even)
        roff[r] = IX(g, ir0, jw, 0);
        c3l[r] = rok[r] ? g.cn3l[jw] : 0.0f;
        c3s[r] = rok[r] ? g.cn3s[jw] : 0.0f;
        cB[r] = (!CN1K && rok[r]) ? g.cnB[jw] : 0.0f;
    }
    // the lane's two columns (x = 2l + c)
    float c2l0, c2l1, c2s0, c2s1, cA0, cA1;
    int fl0, fl1;  // bit 0: 1 <= i <= im, 1: i == 1, 2: i == im, 3: x inside the tile
    {
        auto col = [&](int c, float &cl, float &cs, float &ca, int &fl) {
            const int x = c + 2 * lane, i = ir0 + x;
            const bool ok = (i >= 1 && i <= im);
            cl = ok ? g.cn2l[i] : 0.0f;
            cs = ok ? g.cn2s[i] : 0.0f;
            ca = (!CN1K && ok) ? g.cnA[i] : 0.0f;
            fl = (ok ? 1 : 0) | (i == 1 ? 2 : 0) | (i == im ? 4 : 0) | ((x >= R && x < R + TX) ? 8 : 0);
        };
        col(0, c2l0, c2s0, cA0, fl0);
        col(1, c2l1, c2s1, cA1, fl1);
    }
    // register window: w0/w1[r][m] = column 0/1 of owned row r on plane tau+1-m
    float w0[RPW][W], w1[RPW][W];
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int m = 0; m < W; ++m) w0[r][m] = w1[r][m] = 0.0f;
    // reltmp^2 sums of iterations 0, 1, 2 of the pass
    unsigned long long h0 = 0, l0 = 0, h1 = 0, l1 = 0, h2 = 0, l2 = 0;
    int bad = 0;

    auto request = [&](int k) {
        if (k <= ke) {
            float *Pp = P + (k % NS) * RA;
            float *Bp = Bs + (k % NS) * RA;
            const long long ko = pstride * k;
#pragma unroll
            for (int r = 0; r < RPW; ++r)
                if (rok[r]) {
                    const long long src = roff[r] + ko + lane;
                    const int d = ry[r] * kTbRW + dA;
                    tb_cp_async4(Pp + d, pin + src);
                    tb_cp_async4(Pp + d + 16, pin + src + 32);
                    tb_cp_async4(Bp + d, a.rhs + src);
                    tb_cp_async4(Bp + d + 16, a.rhs + src + 32);
                }
        }
        tb_cp_commit();
    };

#pragma unroll
    for (int k = 0; k < D; ++k) request(kb + k);
    const int tau_end = k1 + 2 * T - 1;  // plane k1 is stored at this step
    for (int tau = kb - 1; tau <= tau_end; ++tau) {
        request(tau + 1 + D);
        tb_cp_wait<D>();  // plane tau+1 has landed (this thread's copies)
        __syncthreads();  // ... and everyone's
        const float *Pn = P + ((tau + 1) % NS) * RA;
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
#pragma unroll
            for (int m = W - 1; m > 0; --m) {
                w0[r][m] = w0[r][m - 1];
                w1[r][m] = w1[r][m - 1];
            }
            if (rok[r] && tau + 1 <= ke) {
                w0[r][0] = Pn[ry[r] * kTbRW + lane];
                w1[r][0] = Pn[ry[r] * kTbRW + 32 + lane];
            }
        }
#pragma unroll
        for (int s = 0; s < 2 * T; ++s) {
            const int q = tau - s;
            const int qlo = (kb == 1) ? 1 : kb + s + 1, qhi = (ke == km) ? km : ke - s - 1;
            if (s < nhs && q >= qlo && q <= qhi) {
                const int nrd = s & 1;
                float *Pq = P + (q % NS) * RA;
                const float *Bq = Bs + (q % NS) * RA;
                const float c4l = g.cn4l[q], c4s = g.cn4s[q];
                const float cnq = CN1K ? a.cn1k[q] : 0.0f;
                const float cC = CN1K ? 0.0f : g.cnC[q];
                const bool top = (q == km), bottom = (q == 1);
                const int lo = s + 1;
                const bool qtile = (q >= k0 && q <= k1);
#pragma unroll
                for (int r = 0; r < RPW; ++r) {
                    const int y = ry[r];
                    if (!rok[r] || y < lo || y >= RH - lo) continue;
                    const int par = (jr0 + y + q + nrd + 1 - ir0) & 1;  // column of the colour in my pair
                    // x neighbour held by the adjacent lane: column 1 of lane-1
                    // (par 0, west) or column 0 of lane+1 (par 1, east)
                    const float vsh = par ? w0[r][s + 1] : w1[r][s + 1];
                    const float nb = __shfl_sync(0xffffffffu, vsh, lane + (par ? 1 : -1));
                    const int x = par + 2 * lane;
                    const int fl = par ? fl1 : fl0;
                    if (x < lo || x >= kTbRW - lo || !(fl & 1)) continue;
                    const float pc = par ? w1[r][s + 1] : w0[r][s + 1];
                    const float own = par ? w0[r][s + 1] : w1[r][s + 1];
                    const float pe = (fl & 4) ? pc : (par ? nb : own);
                    const float pw = (fl & 2) ? pc : (par ? own : nb);
                    const int o = y * kTbRW + par * 32 + lane;
                    const float pn = Pq[o + kTbRW];
                    const float ps = Pq[o - kTbRW];
                    const float pu = top ? pc : (par ? w1[r][s] : w0[r][s]);
                    const float pd = bottom ? pc : (par ? w1[r][s + 2] : w0[r][s + 2]);
                    const float cn1 = CN1K ? cnq : 1.0f / ((par ? cA1 : cA0) + cB[r] + cC);
                    const float reltmp =
                        omega * (cn1 * ((par ? c2l1 : c2l0) * pe + (par ? c2s1 : c2s0) * pw + c3l[r] * pn +
                                        c3s[r] * ps + c4l * pu + c4s * pd - (Bq[o] - rhsav)) -
                                 pc);
                    const float nv = pc + reltmp;
                    Pq[o] = nv;
                    if (par)
                        w1[r][s + 1] = nv;
                    else
                        w0[r][s + 1] = nv;
                    if (!redo && qtile && (fl & 8) && y >= R && y < R + ty && jr0 + y <= jm) {
                        if (s < 2)
                            fix_add_nonneg(reltmp * reltmp, h0, l0, bad);
                        else if (s < 4)
                            fix_add_nonneg(reltmp * reltmp, h1, l1, bad);
                        else
                            fix_add_nonneg(reltmp * reltmp, h2, l2, bad);
                    }
                }
            }
        }
        // plane tau+1-2T is final: store the tile part of the owned rows
        const int qs = tau + 1 - 2 * T;
        if (qs >= k0 && qs <= k1) {
            const long long ko = pstride * qs;
#pragma unroll
            for (int r = 0; r < RPW; ++r) {
                const int y = ry[r];
                if (!rok[r] || y < R || y >= R + ty || jr0 + y > jm) continue;
                float *dst = pout + (roff[r] + ko + 2 * lane);
                const bool s0 = (fl0 & 9) == 9, s1 = (fl1 & 9) == 9;
                if (s0 && s1)  // (ir0 + 2l) + 31 is even: 8-byte aligned
                    *reinterpret_cast<float2 *>(dst) = make_float2(w0[r][2 * T], w1[r][2 * T]);
                else if (s0)
                    dst[0] = w0[r][2 * T];
                else if (s1)
                    dst[1] = w1[r][2 * T];
            }
        }
    }
    tb_cp_wait<0>();  // only empty groups can be left

    // per-iteration partial sums, then the last block finishes the pass
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (!redo) {
#pragma unroll
        for (int t = 0; t < T; ++t) {
            __syncthreads();
            const unsigned long long hi = t == 0 ? h0 : (t == 1 ? h1 : h2), lo = t == 0 ? l0 : (t == 1 ? l1 : l2);
            const i128 v = (i128)(((unsigned __int128)hi << 64) | (unsigned __int128)lo);
            block_fix_sum_any(v, bad, &a.part[b * kTbTMax + t]);
        }
    }
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this block's partials and p stores before its ticket
        s_last = (atomicAdd(&sc->ticket, 1u) == (unsigned)nblocks - 1u);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) sc->ticket = 0u;
    if (redo) {
        if (threadIdx.x == 0) {
            sc->redo = 0;
            sc->pbuf ^= 1;
        }
        return;
    }
    tb_finish_pass(a.part, nblocks, nit, a.pjuge, sc);
}

}  // namespace
}  // namespace les
