// les_sor1.cuh -- one red-black SOR iteration per pass over HBM (T = 1),
// laid out for the issue rate.
//
// Same decomposition as k_sor_tb<1> (les_sor_tb.cuh): a CTA of RH warps owns
// a 128-column x RH-row region of (i,j) columns around a 120 x (RH-4) tile,
// a chunk of k with a two-plane ring, lane l the columns 4l..4l+3 of its
// warp's row, and marches the planes upward with the two colours skewed by
// one plane: at step tau colour 0 (nrd = 0) is swept on plane tau and
// colour 1 on plane tau-1, so one barrier per plane orders everything (the
// argument is written out at k_sor_tb).  What differs is how little work a
// step carries besides the updates:
//   - the plane loop is unrolled by the length of the per-column register
//     window (4 planes), so the window rotates by renaming, not by moves;
//   - the colour's x parity at the first step is warp-uniform, so the loop
//     is compiled once for each parity and every step inside knows which
//     two of its four columns it updates;
//   - the k ghosts (boundp2: p(i,j,0) = p(i,j,1), p(i,j,km+1) = p(i,j,km),
//     press.f95:87-115) need no select: within one iteration the ghost of a
//     cell equals that cell's value before its own update, which is its
//     input value, so the window entry below plane 1 and above plane km is
//     filled with that plane's input values;
//   - only the i ghosts of blocks touching i = 1 or i = im take selects
//     (the EDGE variant);
//   - the residual sum of a pass that is not the step's last iteration is
//     an FP32 sum with a rigorous lower bound (tb_finish_fast).
#pragma once
#include <type_traits>

#include "les_sor_tb.cuh"

namespace les {
namespace {

constexpr int kS1Depth = 2;                       // planes requested ahead of the incoming one
constexpr int kS1NS = 4 + kS1Depth;               // plane slots (p and rhs each)
// p and rhs slots, then per slot the input copies of the two rows that meet
// across the periodic j boundary (odd jm)
__host__ __device__ inline size_t s1_smem(int ty) {
    return sizeof(float) * 2 * (size_t)kTbRW * tb_rh(1, ty) * kS1NS + sizeof(float) * 2 * (size_t)kTbRW * kS1NS;
}

template <int V>
using IC = std::integral_constant<int, V>;

// One pass of one SOR iteration.  blockDim.x = 32 * (ty + 4): warp y owns
// region row y, the real row jw (periodic), whose colour parity is that of
// jw.  JODD (odd jm): rows jm and 1 are j-neighbours of the same colour, and in
// press.f95 each reads the other through the ghost rows 0 and jm+1, which
// boundp1 refreshed before the half-sweep -- the other's value before its own
// update, i.e. its input value in a one-iteration pass.  The warps of those
// two rows also copy their input rows into a side pair of rows per plane
// slot, and read each other there (the region holds each real row once:
// ty + 4 <= jm).
template <bool CN1K, bool JODD, bool DD>
__global__ void __launch_bounds__(1024, 1) k_sor1(Geo g, TbArgs a, const __grid_constant__ TbKCoef kq) {
    extern __shared__ float4 smem4[];
    Scal *sc = a.sc;
    if (sc->converged || sc->sor_iters >= a.itmax) return;
    const bool fast = a.fast && !sc->exact_sums && sc->sor_iters + 1 < a.itmax;
    constexpr int RX = tb_ringx(1), TX = tb_tx(1), NS = kS1NS, D = kS1Depth, RW4 = kTbRW / 4;
    const int ty = a.ty, RH = ty + 4, RA4 = RW4 * RH;
    float4 *P = smem4;          // NS plane slots of p
    float4 *Bs = P + NS * RA4;  // NS plane slots of rhs
    float4 *Sd = Bs + NS * RA4;  // NS slots of the input rows jm (row 0) and 1 (row 1), odd jm
    const float *pin = sc->pbuf ? a.pb1 : a.pb0;
    float *pout = sc->pbuf ? a.pb0 : a.pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    const int lane = threadIdx.x & 31, y = threadIdx.x >> 5;
    const int ir0 = 1 + blockIdx.x * TX - RX, jr0 = 1 + blockIdx.y * ty - 2;
    const int k0 = 1 + blockIdx.z * a.kc, k1 = min(km, k0 + a.kc - 1);
    const int kb = max(1, k0 - 2), ke = min(km, k1 + 2);
    const long long pstride = (long long)g.si * g.sj;
    const int jw = ((jr0 + y - 1) % jm + jm) % jm + 1;  // periodic j
    const bool wrapn = JODD && jw == jm, wraps = JODD && jw == 1;  // j+1 resp. j-1 across the boundary
    const long long coff = IX(g, ir0, jw, 0) + kTbCW * lane;
    const float c3l = g.cn3l[jw], c3s = g.cn3s[jw], cB = CN1K ? 0.0f : g.cnB[jw];
    const bool ytile = (y >= 2 && y < 2 + ty && jr0 + y <= jm);
    const bool row0 = (y >= 1 && y < RH - 1), row1 = (y >= 2 && y < RH - 2);  // rows each colour sweeps
    float c2l[kTbCW], c2s[kTbCW], cA[kTbCW];
    int fl[kTbCW];  // bit 0: 1 <= i <= im, 1: i == 1, 2: i == im, 3 (DD): summed (olo <= i <= ohi)
#pragma unroll
    for (int c = 0; c < kTbCW; ++c) {
        const int i = ir0 + kTbCW * lane + c;
        const bool ok = (i >= 1 && i <= im);
        c2l[c] = ok ? g.cn2l[i] : 0.0f;
        c2s[c] = ok ? g.cn2s[i] : 0.0f;
        cA[c] = (!CN1K && ok) ? g.cnA[i] : 0.0f;
        fl[c] = (ok ? 1 : 0) | (i == 1 ? 2 : 0) | (i == im ? 4 : 0) | ((DD && ok && i >= g.olo && i <= g.ohi) ? 8 : 0);
    }
    const int x0 = kTbCW * lane;
    const bool lane_tile = (x0 >= RX && x0 < RX + TX);
    const bool acc_cells = ytile && lane_tile;
    // x parity of the colour-0 columns at the first step (tau = kb)
    const int par0 = (jw + 1 - ir0 + kb) & 1;

    const int d0 = y * RW4 + lane;
    const float *gsrc = pin + coff, *bsrc = a.rhs + coff;
    auto request = [&](int k, int slot) {
        if (k <= ke) {
            tb_cp_async16(reinterpret_cast<float *>(P + slot * RA4 + d0), gsrc + pstride * k);
            tb_cp_async16(reinterpret_cast<float *>(Bs + slot * RA4 + d0), bsrc + pstride * k);
            if (wrapn || wraps)  // row jm -> side row 0, row 1 -> side row 1
                tb_cp_async16(reinterpret_cast<float *>(Sd + (2 * slot + (wraps ? 1 : 0)) * RW4 + lane),
                              gsrc + pstride * k);
        }
        tb_cp_commit();
    };
    // planes kb .. kb+D-1 in flight, then plane kb waited for
#pragma unroll
    for (int q = 0; q <= D; ++q) request(kb + q, q);
    tb_cp_wait<D>();
    __syncthreads();
    // window w[x][c]: column c of the plane whose step phase is x (planes
    // tau+1, tau, tau-1, tau-2 sit at phases m+1, m, m-1, m-2 of step m)
    float w[4][kTbCW];
    {
        const float4 v = P[d0];  // plane kb, slot 0
        w[0][0] = v.x, w[0][1] = v.y, w[0][2] = v.z, w[0][3] = v.w;
#pragma unroll
        for (int c = 0; c < kTbCW; ++c) {
            w[3][c] = w[0][c];  // plane kb-1: the bottom ghost (kb = 1) or a ring plane
            w[1][c] = 0.0f;
            w[2][c] = 0.0f;
        }
    }
    unsigned long long fh = 0, flo = 0;
    int bad = 0;
    float fsum = 0.0f;
    const int tau_end = k1 + 1;  // plane k1 is stored at this step
    // (DD: and tiles with columns outside the summed ones olo..ohi, whose sums test fl bit 3)
    const bool edge = ir0 <= 1 || ir0 + kTbRW - 1 >= im || (DD && (ir0 + RX < g.olo || ir0 + RX + TX - 1 > g.ohi));

    // Steps kb .. tau_end, four per group.  PAR: colour-0 x parity at the
    // group's first step; FAST: FP32 residual; EDGE: i ghosts by select.
    auto run = [&](auto PARc, auto FASTc, auto EDGEc) {
        constexpr int PAR = decltype(PARc)::value;
        constexpr bool FAST = decltype(FASTc)::value, EDGE = decltype(EDGEc)::value;
        int slot1 = 1;  // slot of plane tau+1
        for (int tau0 = kb; tau0 <= tau_end; tau0 += 4) {
            auto step = [&](auto Mc) {
                constexpr int m = decltype(Mc)::value;
                constexpr int XN = (m + 1) & 3, XC = m & 3, XD = (m + 3) & 3, XDD = (m + 2) & 3;
                constexpr int C0 = (PAR + m) & 1;  // columns C0, C0+2 take both half-sweeps' updates
                const int tau = tau0 + m;
                if (tau > tau_end) return;
                const int sq1 = slot1, sq0 = slot1 == 0 ? NS - 1 : slot1 - 1, sqm = sq0 == 0 ? NS - 1 : sq0 - 1;
                int sreq = slot1 + D;
                if (sreq >= NS) sreq -= NS;
                request(tau + 1 + D, sreq);
                tb_cp_wait<D>();
                __syncthreads();
                // incoming plane tau+1 (above ke: the top ghost, or a ring plane)
                if (tau + 1 <= ke) {
                    const float4 v = P[sq1 * RA4 + d0];
                    w[XN][0] = v.x, w[XN][1] = v.y, w[XN][2] = v.z, w[XN][3] = v.w;
                } else {
#pragma unroll
                    for (int c = 0; c < kTbCW; ++c) w[XN][c] = w[XC][c];
                }
                auto upd = [&](float &pc_ref, float west, float east, float pn, float ps, float pu, float pd, float b,
                               float c4l, float c4s, float cnq, float cC, int C, bool acc) {
                    const float pc = pc_ref;
                    const float pe = (EDGE && (fl[C] & 4)) ? pc : east;
                    const float pw = (EDGE && (fl[C] & 2)) ? pc : west;
                    const float cn1 = CN1K ? cnq : 1.0f / (cA[C] + cB + cC);
                    const float reltmp = omega * (cn1 * (c2l[C] * pe + c2s[C] * pw + c3l * pn + c3s * ps +
                                                         c4l * pu + c4s * pd - (b - rhsav)) -
                                                  pc);
                    pc_ref = pc + reltmp;
                    if (acc && (!EDGE || (fl[C] & (DD ? 8 : 1)))) {
                        const float t2 = reltmp * reltmp;
                        if constexpr (FAST)
                            fsum += t2;
                        else
                            fix_add_nonneg(t2, fh, flo, bad);
                    }
                };
                // colour 0 on plane tau
                if (row0 && tau <= ke) {
                    const float4 *Pq = P + sq0 * RA4 + d0;
                    const float4 nn = wrapn ? Sd[(2 * sq0 + 1) * RW4 + lane] : Pq[RW4];
                    const float4 ss = wraps ? Sd[2 * sq0 * RW4 + lane] : Pq[-RW4];
                    const float4 bb = Bs[sq0 * RA4 + d0];
                    const float c4l = kq.c4l[tau], c4s = kq.c4s[tau];
                    const float cnq = CN1K ? kq.cnk[tau] : 0.0f, cC = CN1K ? 0.0f : g.cnC[tau];
                    const bool acc = acc_cells && tau >= k0 && tau <= k1;
                    if constexpr (C0 == 0) {
                        const float nb = __shfl_sync(0xffffffffu, w[XC][3], lane - 1);
                        upd(w[XC][0], nb, w[XC][1], nn.x, ss.x, w[XN][0], w[XD][0], bb.x, c4l, c4s, cnq, cC, 0, acc);
                        upd(w[XC][2], w[XC][1], w[XC][3], nn.z, ss.z, w[XN][2], w[XD][2], bb.z, c4l, c4s, cnq, cC, 2,
                            acc);
                    } else {
                        const float nb = __shfl_sync(0xffffffffu, w[XC][0], lane + 1);
                        upd(w[XC][1], w[XC][0], w[XC][2], nn.y, ss.y, w[XN][1], w[XD][1], bb.y, c4l, c4s, cnq, cC, 1,
                            acc);
                        upd(w[XC][3], w[XC][2], nb, nn.w, ss.w, w[XN][3], w[XD][3], bb.w, c4l, c4s, cnq, cC, 3, acc);
                    }
                    // publish (the colour-1 columns are rewritten with the same bits)
                    P[sq0 * RA4 + d0] = make_float4(w[XC][0], w[XC][1], w[XC][2], w[XC][3]);
                }
                // colour 1 on plane tau-1: the same x parity as colour 0 on plane tau
                const int q = tau - 1;
                if (row1 && q >= kb) {
                    const float4 *Pq = P + sqm * RA4 + d0;
                    const float4 nn = wrapn ? Sd[(2 * sqm + 1) * RW4 + lane] : Pq[RW4];
                    const float4 ss = wraps ? Sd[2 * sqm * RW4 + lane] : Pq[-RW4];
                    const float4 bb = Bs[sqm * RA4 + d0];
                    const float c4l = kq.c4l[q], c4s = kq.c4s[q];
                    const float cnq = CN1K ? kq.cnk[q] : 0.0f, cC = CN1K ? 0.0f : g.cnC[q];
                    const bool acc = acc_cells && q >= k0 && q <= k1;
                    if constexpr (C0 == 0) {
                        const float nb = __shfl_sync(0xffffffffu, w[XD][3], lane - 1);
                        upd(w[XD][0], nb, w[XD][1], nn.x, ss.x, w[XC][0], w[XDD][0], bb.x, c4l, c4s, cnq, cC, 0, acc);
                        upd(w[XD][2], w[XD][1], w[XD][3], nn.z, ss.z, w[XC][2], w[XDD][2], bb.z, c4l, c4s, cnq, cC, 2,
                            acc);
                    } else {
                        const float nb = __shfl_sync(0xffffffffu, w[XD][0], lane + 1);
                        upd(w[XD][1], w[XD][0], w[XD][2], nn.y, ss.y, w[XC][1], w[XDD][1], bb.y, c4l, c4s, cnq, cC, 1,
                            acc);
                        upd(w[XD][3], w[XD][2], nb, nn.w, ss.w, w[XC][3], w[XDD][3], bb.w, c4l, c4s, cnq, cC, 3, acc);
                    }
                    // plane tau-1 is final: store the tile part of the row
                    if (acc_cells && q >= k0 && q <= k1) {
                        float *dst = pout + (coff + pstride * q);
                        if (!EDGE || (fl[3] & fl[0] & 1))
                            *reinterpret_cast<float4 *>(dst) = make_float4(w[XD][0], w[XD][1], w[XD][2], w[XD][3]);
                        else {
#pragma unroll
                            for (int c = 0; c < kTbCW; ++c)
                                if (fl[c] & 1) dst[c] = w[XD][c];
                        }
                    }
                }
                slot1 = slot1 + 1 == NS ? 0 : slot1 + 1;
            };
            step(IC<0>());
            step(IC<1>());
            step(IC<2>());
            step(IC<3>());
        }
    };
    using True = std::true_type;
    using False = std::false_type;
#define S1_RUN(F, E)                    \
    do {                                \
        if (par0)                       \
            run(IC<1>(), F(), E());     \
        else                            \
            run(IC<0>(), F(), E());     \
    } while (0)
    if (fast) {
        if (edge)
            S1_RUN(True, True);
        else
            S1_RUN(True, False);
    } else {
        if (edge)
            S1_RUN(False, True);
        else
            S1_RUN(False, False);
    }
#undef S1_RUN
    tb_cp_wait<0>();

    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    __syncthreads();
    if (fast) {
        const float v = block_float_sum0(fsum);
        if (threadIdx.x == 0) {
            FixPart fp{};
            fp.lo = __float_as_uint(v);
            a.part[b * kTbTMax] = fp;
        }
    } else {
        const i128 v = (i128)(((unsigned __int128)fh << 64) | (unsigned __int128)flo);
        block_fix_sum_any(v, bad, &a.part[b * kTbTMax]);
    }
    if (DD) return;  // a rank of an x-decomposed domain: the host sums the partials over the ranks
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
    if (fast)
        tb_finish_fast(a.part, nblocks, a.pjuge, sc);
    else
        tb_finish_pass(a.part, nblocks, 1, a.pjuge, sc);
}

}  // namespace
}  // namespace les

namespace les {
namespace {

// ---- two iterations per pass (T = 2) ----------------------------------------
// The layout of k_sor1 with a four-row, four-plane ring (the region shrinks
// by one per half-sweep): at step tau half-sweep s works on plane tau-s, the
// colours of iteration 1 (s = 0, 1) and then of iteration 2 (s = 2, 3), all
// four on the same x parity; each half-sweep publishes its row, and plane
// tau-3 is final after s = 3.  The window holds planes tau+1 .. tau-4 (six),
// so the loop is unrolled by six.  One plane of p and rhs is requested one
// step ahead: seven plane slots, 168 KB at 24 rows.  Iteration 2's k ghosts
// take the cell's own value by select (its ghost is the value after
// iteration 1); iteration 1's come from the window as in k_sor1.  A pass
// that is not the step's last takes FP32 residual sums with the bound of
// tb_finish_fast for each of its iterations.  nit = 1 (an odd last pass,
// the redo of a pass that converged after its first iteration, or the spare
// pass) runs the first two half-sweeps only.  At most 24 rows (768 threads,
// 80 registers: the six-plane window does not fit in 64).
constexpr int kS2Depth = 1, kS2NS = 6 + kS2Depth;
__host__ __device__ inline size_t s2_smem(int ty) {
    return sizeof(float) * 2 * (size_t)kTbRW * tb_rh(2, ty) * kS2NS;
}

// Stop test of a fast (FP32-summed) pass of nit iterations: all counted if
// every iteration's lower bound rules the stop out, else none and exact
// sums for the rest of the step (the next pass repeats from the unchanged
// input buffer).  See tb_finish_fast for the bound.
__device__ void s2_finish_fast(const FixPart *part, int nblocks, int nit, float pjuge, Scal *s) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) s_ok = 1;
    __syncthreads();
    for (int t = 0; t < nit; ++t) {
        float v = 0.0f;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
            v += __uint_as_float((unsigned)__ldcg(&part[(size_t)b * kTbTMax + t].lo));
        v = block_float_sum0(v);
        if (threadIdx.x == 0) {
            const float lb = __fsub_rd(__fmul_rd(v, 0.99609375f), 0x1p-33f);
            if (!(lb >= pjuge && lb < 0x1p40f)) s_ok = 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (s_ok) {
            s->sor_iters += nit;
            s->pbuf ^= 1;
        } else {
            s->exact_sums = 1;
        }
    }
}

template <bool CN1K>
__global__ void __launch_bounds__(768, 1) k_sor2(Geo g, TbArgs a, const __grid_constant__ TbKCoef kq) {
    extern __shared__ float4 smem4[];
    Scal *sc = a.sc;
    const bool redo = (a.mode == 1);
    if (!redo && (sc->converged || sc->sor_iters >= a.itmax)) return;
    const int nit = redo ? sc->redo : min(a.niter, a.itmax - sc->sor_iters);
    if (nit <= 0) return;
    const bool fast = a.fast && !redo && !sc->exact_sums && sc->sor_iters + nit < a.itmax;
    constexpr int RX = tb_ringx(2), TX = tb_tx(2), NS = kS2NS, D = kS2Depth, RW4 = kTbRW / 4;
    const int ty = a.ty, RH = ty + 8, RA4 = RW4 * RH;
    float4 *P = smem4;
    float4 *Bs = P + NS * RA4;
    const float *pin = sc->pbuf ? a.pb1 : a.pb0;
    float *pout = sc->pbuf ? a.pb0 : a.pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    const int lane = threadIdx.x & 31, y = threadIdx.x >> 5;
    const int ir0 = 1 + blockIdx.x * TX - RX, jr0 = 1 + blockIdx.y * ty - 4;
    const int k0 = 1 + blockIdx.z * a.kc, k1 = min(km, k0 + a.kc - 1);
    const int kb = max(1, k0 - 4), ke = min(km, k1 + 4);
    const long long pstride = (long long)g.si * g.sj;
    const int jw = ((jr0 + y - 1) % jm + jm) % jm + 1;
    const long long coff = IX(g, ir0, jw, 0) + kTbCW * lane;
    const float c3l = g.cn3l[jw], c3s = g.cn3s[jw], cB = CN1K ? 0.0f : g.cnB[jw];
    const bool ytile = (y >= 4 && y < 4 + ty && jr0 + y <= jm);
    float c2l[kTbCW], c2s[kTbCW], cA[kTbCW];
    int fl[kTbCW];
#pragma unroll
    for (int c = 0; c < kTbCW; ++c) {
        const int i = ir0 + kTbCW * lane + c;
        const bool ok = (i >= 1 && i <= im);
        c2l[c] = ok ? g.cn2l[i] : 0.0f;
        c2s[c] = ok ? g.cn2s[i] : 0.0f;
        cA[c] = (!CN1K && ok) ? g.cnA[i] : 0.0f;
        fl[c] = (ok ? 1 : 0) | (i == 1 ? 2 : 0) | (i == im ? 4 : 0);
    }
    const int x0 = kTbCW * lane;
    const bool lane_tile = (x0 >= RX && x0 < RX + TX);
    const bool acc_cells = !redo && ytile && lane_tile;
    const int par0 = (jr0 + y + 1 - ir0 + kb) & 1;

    const int d0 = y * RW4 + lane;
    const float *gsrc = pin + coff, *bsrc = a.rhs + coff;
    auto request = [&](int k, int slot) {
        if (k <= ke) {
            tb_cp_async16(reinterpret_cast<float *>(P + slot * RA4 + d0), gsrc + pstride * k);
            tb_cp_async16(reinterpret_cast<float *>(Bs + slot * RA4 + d0), bsrc + pstride * k);
        }
        tb_cp_commit();
    };
#pragma unroll
    for (int q = 0; q <= D; ++q) request(kb + q, q);
    tb_cp_wait<D>();
    __syncthreads();
    // window: w[x][c], plane kb + x' at phase x' mod 6
    float w[6][kTbCW];
    {
        const float4 v = P[d0];
        w[0][0] = v.x, w[0][1] = v.y, w[0][2] = v.z, w[0][3] = v.w;
#pragma unroll
        for (int c = 0; c < kTbCW; ++c) {
            w[1][c] = 0.0f;
            w[2][c] = w[0][c];  // planes kb-4 .. kb-1: the bottom ghost (kb = 1) or ring planes
            w[3][c] = w[0][c];
            w[4][c] = w[0][c];
            w[5][c] = w[0][c];
        }
    }
    float fs0 = 0.0f, fs1 = 0.0f;  // FP32 residual sums of iterations 1 and 2
    unsigned long long h0 = 0, l0 = 0, h1 = 0, l1 = 0;
    int bad = 0;
    const int tau_end = k1 + (nit == 2 ? 3 : 1);
    const bool edge = ir0 <= 1 || ir0 + kTbRW - 1 >= im;

    auto run = [&](auto PARc, auto FASTc, auto EDGEc, auto NITc) {
        constexpr int PAR = decltype(PARc)::value, NIT = decltype(NITc)::value;
        constexpr bool FAST = decltype(FASTc)::value, EDGE = decltype(EDGEc)::value;
        int slot1 = 1;  // slot of plane tau+1
        for (int tau0 = kb; tau0 <= tau_end; tau0 += 6) {
            auto step = [&](auto Mc) {
                constexpr int m = decltype(Mc)::value;
                constexpr int C0 = (PAR + m) & 1;
                // window phases of planes tau+1, tau, tau-1, .., tau-4
                constexpr int XP1 = (m + 1) % 6, X0 = m % 6, X1 = (m + 5) % 6, X2 = (m + 4) % 6,
                              X3 = (m + 3) % 6;
                const int tau = tau0 + m;
                if (tau > tau_end) return;
                int sq[4];  // slots of planes tau, tau-1, tau-2, tau-3
                sq[0] = slot1 == 0 ? NS - 1 : slot1 - 1;
#pragma unroll
                for (int s = 1; s < 4; ++s) sq[s] = sq[s - 1] == 0 ? NS - 1 : sq[s - 1] - 1;
                int sreq = slot1 + D;
                if (sreq >= NS) sreq -= NS;
                request(tau + 1 + D, sreq);
                tb_cp_wait<D>();
                __syncthreads();
                if (tau + 1 <= ke) {
                    const float4 v = P[slot1 * RA4 + d0];
                    w[XP1][0] = v.x, w[XP1][1] = v.y, w[XP1][2] = v.z, w[XP1][3] = v.w;
                } else {
#pragma unroll
                    for (int c = 0; c < kTbCW; ++c) w[XP1][c] = w[X0][c];
                }
                // half-sweep s on plane q = tau - s: the cell's window row XQ, its
                // neighbours above (XU) and below (XD)
                auto half = [&](auto Sc, auto XQc, auto XUc, auto XDc) {
                    constexpr int S = decltype(Sc)::value, XQ = decltype(XQc)::value, XU = decltype(XUc)::value,
                                  XD = decltype(XDc)::value;
                    const int q = tau - S;
                    if (!(q >= kb && q <= ke && y >= S + 1 && y < RH - S - 1)) return;
                    const float4 *Pq = P + sq[S] * RA4 + d0;
                    const float4 nn = Pq[RW4], ss = Pq[-RW4], bb = Bs[sq[S] * RA4 + d0];
                    const float c4l = kq.c4l[q], c4s = kq.c4s[q];
                    const float cnq = CN1K ? kq.cnk[q] : 0.0f, cC = CN1K ? 0.0f : g.cnC[q];
                    const bool acc = acc_cells && q >= k0 && q <= k1;
                    const bool top = S >= 2 && q == km, bot = S >= 2 && q == 1;
                    auto upd = [&](auto Cc, float west, float east, float pn, float ps, float b) {
                        constexpr int C = decltype(Cc)::value;
                        const float pc = w[XQ][C];
                        const float pe = (EDGE && (fl[C] & 4)) ? pc : east;
                        const float pw = (EDGE && (fl[C] & 2)) ? pc : west;
                        const float pu = top ? pc : w[XU][C];
                        const float pd = bot ? pc : w[XD][C];
                        const float cn1 = CN1K ? cnq : 1.0f / (cA[C] + cB + cC);
                        const float reltmp = omega * (cn1 * (c2l[C] * pe + c2s[C] * pw + c3l * pn + c3s * ps +
                                                             c4l * pu + c4s * pd - (b - rhsav)) -
                                                      pc);
                        w[XQ][C] = pc + reltmp;
                        if (acc && (!EDGE || (fl[C] & 1))) {
                            const float t2 = reltmp * reltmp;
                            if constexpr (FAST) {
                                if (S < 2)
                                    fs0 += t2;
                                else
                                    fs1 += t2;
                            } else {
                                if (S < 2)
                                    fix_add_nonneg(t2, h0, l0, bad);
                                else
                                    fix_add_nonneg(t2, h1, l1, bad);
                            }
                        }
                    };
                    if constexpr (C0 == 0) {
                        const float nb = __shfl_sync(0xffffffffu, w[XQ][3], lane - 1);
                        upd(IC<0>(), nb, w[XQ][1], nn.x, ss.x, bb.x);
                        upd(IC<2>(), w[XQ][1], w[XQ][3], nn.z, ss.z, bb.z);
                    } else {
                        const float nb = __shfl_sync(0xffffffffu, w[XQ][0], lane + 1);
                        upd(IC<1>(), w[XQ][0], w[XQ][2], nn.y, ss.y, bb.y);
                        upd(IC<3>(), w[XQ][2], nb, nn.w, ss.w, bb.w);
                    }
                    if (S < 2 * NIT - 1)  // later half-sweeps of the pass read this row
                        P[sq[S] * RA4 + d0] = make_float4(w[XQ][0], w[XQ][1], w[XQ][2], w[XQ][3]);
                };
                half(IC<0>(), IC<X0>(), IC<XP1>(), IC<X1>());
                half(IC<1>(), IC<X1>(), IC<X0>(), IC<X2>());
                if constexpr (NIT == 2) {
                    half(IC<2>(), IC<X2>(), IC<X1>(), IC<X3>());
                    half(IC<3>(), IC<X3>(), IC<X2>(), IC<(m + 2) % 6>());  // below: plane tau-4
                }
                // the pass's last half-sweep finished plane qs: store its tile part
                constexpr int XS = NIT == 2 ? X3 : X1;
                const int qs = tau - (2 * NIT - 1);
                if (acc_cells || (redo && ytile && lane_tile)) {
                    if (qs >= k0 && qs <= k1) {
                        float *dst = pout + (coff + pstride * qs);
                        if (!EDGE || (fl[3] & fl[0] & 1))
                            *reinterpret_cast<float4 *>(dst) = make_float4(w[XS][0], w[XS][1], w[XS][2], w[XS][3]);
                        else {
#pragma unroll
                            for (int c = 0; c < kTbCW; ++c)
                                if (fl[c] & 1) dst[c] = w[XS][c];
                        }
                    }
                }
                slot1 = slot1 + 1 == NS ? 0 : slot1 + 1;
            };
            step(IC<0>());
            step(IC<1>());
            step(IC<2>());
            step(IC<3>());
            step(IC<4>());
            step(IC<5>());
        }
    };
    using True = std::true_type;
    using False = std::false_type;
#define S2_RUN(F, E, N)                         \
    do {                                        \
        if (par0)                               \
            run(IC<1>(), F(), E(), IC<N>());    \
        else                                    \
            run(IC<0>(), F(), E(), IC<N>());    \
    } while (0)
    if (nit == 2) {
        if (fast) {
            if (edge) S2_RUN(True, True, 2);
            else S2_RUN(True, False, 2);
        } else {
            if (edge) S2_RUN(False, True, 2);
            else S2_RUN(False, False, 2);
        }
    } else {
        if (fast) {
            if (edge) S2_RUN(True, True, 1);
            else S2_RUN(True, False, 1);
        } else {
            if (edge) S2_RUN(False, True, 1);
            else S2_RUN(False, False, 1);
        }
    }
#undef S2_RUN
    tb_cp_wait<0>();

    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    __syncthreads();
    if (!redo) {
        if (fast) {
            const float v0 = block_float_sum0(fs0);
            __syncthreads();
            const float v1 = block_float_sum0(fs1);
            if (threadIdx.x == 0) {
                FixPart f0{}, f1{};
                f0.lo = __float_as_uint(v0);
                f1.lo = __float_as_uint(v1);
                a.part[b * kTbTMax] = f0;
                a.part[b * kTbTMax + 1] = f1;
            }
        } else {
            block_fix_sum_any((i128)(((unsigned __int128)h0 << 64) | (unsigned __int128)l0), bad,
                              &a.part[b * kTbTMax]);
            __syncthreads();
            block_fix_sum_any((i128)(((unsigned __int128)h1 << 64) | (unsigned __int128)l1), bad,
                              &a.part[b * kTbTMax + 1]);
        }
    }
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
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
        s2_finish_fast(a.part, nblocks, nit, a.pjuge, sc);
    else
        tb_finish_pass(a.part, nblocks, nit, a.pjuge, sc);
}

}  // namespace
}  // namespace les
