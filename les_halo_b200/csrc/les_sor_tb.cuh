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
//   - a CTA owns a (128 - 4T) x ty tile of (i,j) columns, a chunk of k, and
//     a ring of R = 2T cells (and planes) around them; half-sweep s updates
//     the region shrunk by s+1 on every side, so after 2T half-sweeps the
//     tile holds exact values;
//   - planes march upward: at step tau half-sweep s works on plane tau-s,
//     in order s = 0,1,.., so each plane sees its neighbours at the right
//     level;
//   - a warp owns one region row (128 columns), lane l the columns 4l..4l+3,
//     whose values on the last 2T+2 planes stay in registers; a half-sweep
//     updates two of them (one colour), taking the k neighbours and three
//     of the four x neighbours from registers, the fourth from the adjacent
//     lane (one shuffle), and the j neighbours from a shared copy of the
//     plane (rows stored as x -> (x%4)*32 + x/4, so these reads are
//     bank-conflict free);
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
#include <type_traits>

#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

constexpr int kTbCW = 4;              // columns per lane
constexpr int kTbRW = 32 * kTbCW;     // region row: 128 columns
constexpr int kTbTMax = 3;            // iterations per pass
constexpr int kTbDepth = 2;           // planes requested ahead of the one a step needs
constexpr int kTbMaxRH = 32;          // region rows, one warp each
constexpr int kTbMaxChunks = 8;

__host__ __device__ constexpr int tb_ring(int T) { return 2 * T; }
// ring in x: 2T rounded up to 4 columns, so every row of the region starts
// on a 16-byte boundary (whole float4 per lane)
__host__ __device__ constexpr int tb_ringx(int T) { return (2 * T + 3) / 4 * 4; }
// tile columns: the region minus a ring on each side
__host__ __device__ constexpr int tb_tx(int T) { return kTbRW - 2 * tb_ringx(T); }
// shared plane slots (p and rhs each): 2T planes in work, the incoming one,
// kTbDepth in flight and one of slack so a request never hits a plane a
// slower warp may still read
__host__ __device__ constexpr int tb_ns(int T) { return 2 * T + 2 + kTbDepth; }
__host__ __device__ inline int tb_rh(int T, int ty) { return ty + 2 * tb_ring(T); }
__host__ __device__ inline int tb_warps(int T, int ty) { return tb_rh(T, ty); }
__host__ __device__ inline size_t tb_smem(int T, int ty) {
    return sizeof(float) * 2 * (size_t)kTbRW * tb_rh(T, ty) * tb_ns(T);
}
// rows (= warps) within the kernels' launch bounds: 32 for one iteration per
// pass, 24 for more (their longer register windows need more registers)
__host__ __device__ inline bool tb_fits(int T, int ty) {
    return T >= 1 && T <= kTbTMax && ty >= 1 && tb_rh(T, ty) <= (T == 1 ? kTbMaxRH : 24);
}

struct TbArgs {
    float *pb0, *pb1;         // the two p buffers (Scal::pbuf says which is current)
    const float *rhs;         // raw rhs (rhsav not yet subtracted)
    const float *cn1k;        // cn1 per k when it depends on k only
    int ty, kc, niter, mode;  // tile rows, planes per k chunk, iterations, 0 pass / 1 redo
    int itmax;                // iterations of the step (nmaxp): a pass starting at itmax does nothing
    int fast;                 // one-iteration passes may take the FP32 stop test (tb_finish_fast)
    float pjuge;              // stop threshold (press.f95:107)
    FixPart *part;            // kTbTMax partial sums per block
    Scal *sc;
};

// Per-plane coefficients of the SOR update, passed by value as a
// __grid_constant__ kernel parameter: a warp-uniform plane index reads them
// from the constant bank without address arithmetic or a global load.
// Index q = 1..km; grids with km >= kTbKMax use the per-colour sweeps.
constexpr int kTbKMax = 1024;
struct TbKCoef {
    float c4l[kTbKMax], c4s[kTbKMax];  // cn4l(q), cn4s(q)
    float cnk[kTbKMax];                // cn1 by plane when it depends on k only (CN1K)
};

// Exact Q63.64 term (les_fix.h) of a non-negative float below 2^62: the
// integer part and the fraction scaled by 2^64, both exact in FP64.  A term
// below 1 is the fraction alone, and x * 2^64 is then exact in FP32 (a
// power-of-two scaling inside the normal range), so one truncating
// conversion gives it.
__device__ __forceinline__ void fix_add_nonneg(float x, unsigned long long &hi, unsigned long long &lo, int &bad) {
    unsigned long long fr, ip;
    if (x < 1.0f) {
        fr = __float2ull_rz(x * 18446744073709551616.0f);
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

// Sum of v over a block of whole warps, returned to thread 0: shuffles
// within each warp, then thread 0 adds the warp sums in order.  Adds on any
// leaf-to-root path: 5 + warps.
__device__ __forceinline__ float block_float_sum0(float v) {
    __shared__ float s_f[32];
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) s_f[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_f[w];
    return t;
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

__device__ __forceinline__ void tb_cp_async16(float *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
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

// FP32 stop test of a one-iteration pass that is not the step's last
// iteration.  The exact test of press.f95:114 is sor < pjuge with sor the
// exact sum S_x of the terms t = fl(reltmp^2) (each truncated to 2^-64,
// les_fix.h) rounded to FP32.  Here the terms were summed in FP32 along a
// tree with at most d adds from any term to the root (per thread 4 per
// plane, block_float_sum0 twice, and the strided pass below; the host
// keeps d <= 2^16).  With round-to-nearest on non-negative numbers the
// computed sum v <= (1+u)^d * sum(t), u = 2^-24, so
//     S_x >= v * (1 - d u) - n 2^-64 >= v * (1 - 2^-8) - 2^-33  (n < 2^31 cells),
// evaluated below with rounding toward -inf as lb.  If pjuge <= lb < 2^40
// then S_x >= lb, no exact partial overflows, and rounding S_x to FP32
// gives at least lb (lb is an FP32 number): the exact test would not stop
// either.  The iteration is then counted and its output buffer becomes
// current.  Otherwise (possibly converged, or NaN/inf/huge sums) nothing is
// counted, the buffers stay as they were, and every later pass of the step
// sums exactly: the next launch repeats this iteration from the unchanged
// input buffer (a pass reads one buffer and writes the other), so the
// decision, the reported residual and p are those of exact sums.
__device__ void tb_finish_fast(const FixPart *part, int nblocks, float pjuge, Scal *s) {
    float v = 0.0f;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        v += __uint_as_float((unsigned)__ldcg(&part[(size_t)b * kTbTMax].lo));
    v = block_float_sum0(v);
    if (threadIdx.x == 0) {
        const float lb = __fsub_rd(__fmul_rd(v, 0.99609375f), 0x1p-33f);
        if (lb >= pjuge && lb < 0x1p40f) {
            s->sor_iters += 1;
            s->pbuf ^= 1;
        } else {
            s->exact_sums = 1;
        }
    }
}

// One pass of niter <= T iterations (mode 0), or the redo of scal->redo
// iterations after a pass that converged part-way (mode 1).
// CN1K: cn1 depends on k only (uniform dx and dy), read from cn1k[k].
// blockDim.x = 32 * tb_rh(T, ty): warp y owns region row y.
template <int T, bool CN1K>
__global__ void __launch_bounds__(T == 1 ? 1024 : 768) k_sor_tb(Geo g, TbArgs a, const __grid_constant__ TbKCoef kq) {
    extern __shared__ float4 smem4[];
    Scal *sc = a.sc;
    const bool redo = (a.mode == 1);
    if (!redo && (sc->converged || sc->sor_iters >= a.itmax)) return;
    // FP32 residual sum for one-iteration passes before the step's last
    // iteration, until a pass cannot decide in FP32 (tb_finish_fast)
    const bool fast = T == 1 && a.fast && !redo && !sc->exact_sums && sc->sor_iters + 1 < a.itmax;
    const int nit = redo ? sc->redo : a.niter;
    if (nit <= 0) return;
    constexpr int R = tb_ring(T), RX = tb_ringx(T), TX = tb_tx(T), NS = tb_ns(T), D = kTbDepth, W = 2 * T + 2;
    constexpr int RW4 = kTbRW / 4;  // float4 per region row
    const int nhs = (T == 1) ? 2 : 2 * nit;  // a one-iteration pass is never a redo
    const int ty = a.ty, RH = ty + 2 * R, RA4 = RW4 * RH;
    float4 *P = smem4;          // NS plane slots of p
    float4 *Bs = P + NS * RA4;  // NS plane slots of rhs
    const float *pin = sc->pbuf ? a.pb1 : a.pb0;
    float *pout = sc->pbuf ? a.pb0 : a.pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    const int lane = threadIdx.x & 31, y = threadIdx.x >> 5;  // warp y owns region row y
    const int ir0 = 1 + blockIdx.x * TX - RX, jr0 = 1 + blockIdx.y * ty - R;
    const int k0 = 1 + blockIdx.z * a.kc, k1 = min(km, k0 + a.kc - 1);
    const int kb = max(1, k0 - R), ke = min(km, k1 + R);
    const long long pstride = (long long)g.si * g.sj;

    const int jw = ((jr0 + y - 1) % jm + jm) % jm + 1;  // periodic j (jm even)
    // box offset of (ir0 + 4*lane, jw, k=0); (ir0 + 31) is a multiple of 4
    const long long coff = IX(g, ir0, jw, 0) + kTbCW * lane;
    const float c3l = g.cn3l[jw], c3s = g.cn3s[jw], cB = CN1K ? 0.0f : g.cnB[jw];
    const bool ytile = (y >= R && y < R + ty && jr0 + y <= jm);
    // the lane's columns x = 4l + c
    float c2l[kTbCW], c2s[kTbCW], cA[kTbCW];
    int fl[kTbCW];  // bit 0: 1 <= i <= im, 1: i == 1, 2: i == im, 3: x inside the tile
#pragma unroll
    for (int c = 0; c < kTbCW; ++c) {
        const int x = kTbCW * lane + c, i = ir0 + x;
        const bool ok = (i >= 1 && i <= im);
        c2l[c] = ok ? g.cn2l[i] : 0.0f;
        c2s[c] = ok ? g.cn2s[i] : 0.0f;
        cA[c] = (!CN1K && ok) ? g.cnA[i] : 0.0f;
        fl[c] = (ok ? 1 : 0) | (i == 1 ? 2 : 0) | (i == im ? 4 : 0) | ((x >= RX && x < RX + TX) ? 8 : 0);
    }
    // the tile's columns come in whole lanes (RX and TX are multiples of 4)
    const bool lane_tile = (fl[0] & 8) != 0;
    const bool acc_cells = !redo && ytile && lane_tile;  // this lane's updates enter the residual
    // x parity of the colour updated at step tau: (pbase + tau) & 1 for every
    // half-sweep (q = tau - s and nrd = s & 1 move together)
    const int pbase = (jr0 + y + 1 - ir0) & 1;
    // register window: w[c][m] = column c on plane tau+1-m
    float w[kTbCW][W];
#pragma unroll
    for (int c = 0; c < kTbCW; ++c)
#pragma unroll
        for (int m = 0; m < W; ++m) w[c][m] = 0.0f;
    // reltmp^2 sums of iterations 0, 1, 2 of the pass
    unsigned long long h0 = 0, l0 = 0, h1 = 0, l1 = 0, h2 = 0, l2 = 0;
    int bad = 0;
    float fsum = 0.0f;  // the FP32 sum of a fast pass

    // plane k of this warp's row: one 16-byte copy per lane and array
    const int d0 = y * RW4 + lane;
    auto request = [&](int k, int slot) {
        if (k <= ke) {
            const long long src = coff + pstride * k;
            tb_cp_async16(reinterpret_cast<float *>(P + slot * RA4 + d0), pin + src);
            tb_cp_async16(reinterpret_cast<float *>(Bs + slot * RA4 + d0), a.rhs + src);
        }
        tb_cp_commit();
    };

#pragma unroll
    for (int k = 0; k < D; ++k) request(kb + k, (kb + k) % NS);
    const int tau_end = k1 + 2 * T - 1;  // plane k1 is stored at this step

    // The plane loop, compiled for each stop test (FAST: the FP32 sum) and
    // for blocks whose region reaches i = 1 or i = im (EDGE).  A half-sweep
    // updates every column of its rows and planes, the ring columns
    // included.  A ring column's update may read a value from outside the
    // region (the lane shuffles wrap around); such values move inward by at
    // most one column per half-sweep, 2T columns in all, and the x ring has
    // RX >= 2T columns, so the tile is exact.  Columns outside 1..im are
    // updated the same way and no cell inside reads them: the ghost
    // neighbour of i = 1 and of i = im is the cell itself (boundp1,
    // press.f95:87-115).  Only tile cells inside the grid enter the residual.
    static_assert(tb_ringx(T) >= 2 * T && tb_ringx(T) % kTbCW == 0 && tb_tx(T) % kTbCW == 0,
                  "the ring must hold 2T columns, and i = 1 must fall on column 0 of a lane");
    const bool edge = ir0 <= 1 || ir0 + kTbRW - 1 >= im;
    auto sweep = [&](auto FASTc, auto EDGEc) {
        constexpr bool FAST = decltype(FASTc)::value, EDGE = decltype(EDGEc)::value;
        int st1 = kb % NS;  // slot of plane tau+1
        for (int tau = kb - 1; tau <= tau_end; ++tau) {
            request(tau + 1 + D, st1 + D >= NS ? st1 + D - NS : st1 + D);
            tb_cp_wait<D>();  // plane tau+1 has landed (this thread's copies)
            __syncthreads();  // ... and everyone's
#pragma unroll
            for (int c = 0; c < kTbCW; ++c)
#pragma unroll
                for (int m = W - 1; m > 0; --m) w[c][m] = w[c][m - 1];
            if (tau + 1 <= ke) {
                const float4 v = P[st1 * RA4 + d0];
                w[0][0] = v.x;
                w[1][0] = v.y;
                w[2][0] = v.z;
                w[3][0] = v.w;
            }
#pragma unroll
            for (int s = 0; s < 2 * T; ++s) {
                const int q = tau - s;
                const int qlo = (kb == 1) ? 1 : kb + s + 1, qhi = (ke == km) ? km : ke - s - 1;  // hoisted by the compiler
                const int lo = s + 1;
                if (s < nhs && q >= qlo && q <= qhi && y >= lo && y < RH - lo) {
                    int sq = st1 - 1 - s;
                    if (sq < 0) sq += NS;
                    float4 *Pq = P + sq * RA4 + d0;
                    const float4 nn = Pq[RW4], ss = Pq[-RW4], bb = Bs[sq * RA4 + d0];
                    const float pn4[kTbCW] = {nn.x, nn.y, nn.z, nn.w}, ps4[kTbCW] = {ss.x, ss.y, ss.z, ss.w};
                    const float b4[kTbCW] = {bb.x, bb.y, bb.z, bb.w};
                    const float c4l = kq.c4l[q], c4s = kq.c4s[q];
                    const float cnq = CN1K ? kq.cnk[q] : 0.0f;
                    const float cC = CN1K ? 0.0f : g.cnC[q];
                    const bool top = (q == km), bottom = (q == 1);
                    const bool acc = acc_cells && q >= k0 && q <= k1;
                    // update column C (of this half-sweep's colour) given its x neighbours
                    auto upd = [&](auto Cc, float west, float east) {
                        constexpr int C = decltype(Cc)::value;
                        const float pc = w[C][s + 1];
                        const float pe = (EDGE && (fl[C] & 4)) ? pc : east;
                        const float pw = (EDGE && C == 0 && (fl[0] & 2)) ? pc : west;
                        const float pu = top ? pc : w[C][s];
                        const float pd = bottom ? pc : w[C][s + 2];
                        const float cn1 = CN1K ? cnq : 1.0f / (cA[C] + cB + cC);
                        const float reltmp = omega * (cn1 * (c2l[C] * pe + c2s[C] * pw + c3l * pn4[C] + c3s * ps4[C] +
                                                             c4l * pu + c4s * pd - (b4[C] - rhsav)) -
                                                      pc);
                        w[C][s + 1] = pc + reltmp;
                        if (acc && (!EDGE || (fl[C] & 1))) {
                            const float t2 = reltmp * reltmp;
                            if constexpr (FAST)
                                fsum += t2;
                            else if (s < 2)
                                fix_add_nonneg(t2, h0, l0, bad);
                            else if (s < 4)
                                fix_add_nonneg(t2, h1, l1, bad);
                            else
                                fix_add_nonneg(t2, h2, l2, bad);
                        }
                    };
                    // x parity of this colour's cells on the row
                    if (((pbase + tau) & 1) == 0) {
                        // cells 4l, 4l+2; the west neighbour of 4l is column 3 of lane-1
                        const float nb = __shfl_sync(0xffffffffu, w[3][s + 1], lane - 1);
                        upd(std::integral_constant<int, 0>(), nb, w[1][s + 1]);
                        upd(std::integral_constant<int, 2>(), w[1][s + 1], w[3][s + 1]);
                    } else {
                        // cells 4l+1, 4l+3; the east neighbour of 4l+3 is column 0 of lane+1
                        const float nb = __shfl_sync(0xffffffffu, w[0][s + 1], lane + 1);
                        upd(std::integral_constant<int, 1>(), w[0][s + 1], w[2][s + 1]);
                        upd(std::integral_constant<int, 3>(), w[2][s + 1], nb);
                    }
                    // publish the row's four columns (the other colour's two are
                    // unchanged, so concurrent readers of those see the same bits)
                    *Pq = make_float4(w[0][s + 1], w[1][s + 1], w[2][s + 1], w[3][s + 1]);
                }
            }
            // plane tau+1-2T is final: store the tile part of the row
            const int qs = tau + 1 - 2 * T;
            if (ytile && lane_tile && qs >= k0 && qs <= k1) {
                float *dst = pout + (coff + pstride * qs);
                if (!EDGE || (fl[3] & 1))  // all four columns inside the grid: one 16-byte store
                    *reinterpret_cast<float4 *>(dst) =
                        make_float4(w[0][2 * T], w[1][2 * T], w[2][2 * T], w[3][2 * T]);
                else {
#pragma unroll
                    for (int c = 0; c < kTbCW; ++c)
                        if (fl[c] & 1) dst[c] = w[c][2 * T];
                }
            }
            st1 = (st1 + 1 == NS) ? 0 : st1 + 1;
        }
    };
    using True = std::true_type;
    using False = std::false_type;
    if (T == 1 && fast) {
        if (edge)
            sweep(True(), True());
        else
            sweep(True(), False());
    } else {
        if (edge)
            sweep(False(), True());
        else
            sweep(False(), False());
    }
    tb_cp_wait<0>();  // only empty groups can be left

    // per-iteration partial sums, then the last block finishes the pass
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (fast) {
        __syncthreads();
        const float v = block_float_sum0(fsum);
        if (threadIdx.x == 0) {
            FixPart fp{};
            fp.lo = __float_as_uint(v);
            a.part[b * kTbTMax] = fp;
        }
    } else if (!redo) {
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
    if (fast)
        tb_finish_fast(a.part, nblocks, a.pjuge, sc);
    else
        tb_finish_pass(a.part, nblocks, nit, a.pjuge, sc);
}

}  // namespace
}  // namespace les
