// les_sor1p.cuh -- the one-iteration SOR pass (k_sor1) with two region rows
// per warp.
//
// Same decomposition, plane march, colour skew, shared-memory slots and
// results as k_sor1 (les_sor1.cuh); warp w owns region rows 2w and 2w+1
// (blockDim.x = 16 * (ty + 4), ty + 4 even), so the per-plane barrier, the
// slot bookkeeping and the loop are shared by eight cells per lane instead of
// four, and each row's neighbour inside the warp comes from registers
// instead of shared memory: row 2w+1 reads row 2w there, row 2w reads row
// 2w+1.  Within a half-sweep every update reads the other colour only,
// except across the periodic j boundary with odd jm, where rows jm and 1
// are neighbours of one colour and each reads the other's value from
// before the half-sweep (k_sor1's comment); the in-warp reads therefore take
// a copy of the neighbour row's values made before the half-sweep's
// updates, which for the other colour are the same values.  Neighbours
// outside the warp come from shared memory, or from the side rows of
// k_sor1 across the boundary with odd jm.
#pragma once
#include "les_sor1.cuh"

namespace les {
namespace {

template <bool CN1K, bool JODD, bool DD>
__global__ void __launch_bounds__(512, 1) k_sor1p(Geo g, TbArgs a, const __grid_constant__ TbKCoef kq) {
    extern __shared__ float4 smem4[];
    Scal *sc = a.sc;
    if (sc->converged || sc->sor_iters >= a.itmax) return;
    const bool fast = a.fast && !sc->exact_sums && sc->sor_iters + 1 < a.itmax;
    constexpr int RX = tb_ringx(1), TX = tb_tx(1), NS = kS1NS, D = kS1Depth, RW4 = kTbRW / 4;
    const int ty = a.ty, RH = ty + 4, RA4 = RW4 * RH;
    float4 *P = smem4;           // NS plane slots of p
    float4 *Bs = P + NS * RA4;   // NS plane slots of rhs
    float4 *Sd = Bs + NS * RA4;  // NS slots of the input rows jm (row 0) and 1 (row 1), odd jm
    const float *pin = sc->pbuf ? a.pb1 : a.pb0;
    float *pout = sc->pbuf ? a.pb0 : a.pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
    const int ir0 = 1 + blockIdx.x * TX - RX, jr0 = 1 + blockIdx.y * ty - 2;
    const int k0 = 1 + blockIdx.z * a.kc, k1 = min(km, k0 + a.kc - 1);
    const int kb = max(1, k0 - 2), ke = min(km, k1 + 2);
    const long long pstride = (long long)g.si * g.sj;
    const int x0 = kTbCW * lane;
    const bool lane_tile = (x0 >= RX && x0 < RX + TX);
    // per row r of the warp (region row y = 2 wy + r, real row jw)
    int jw[2], d0[2];
    bool wrapn[2], wraps[2], row0[2], row1[2], acc_cells[2];
    long long coff[2];
    float c3l[2], c3s[2], cB[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int y = 2 * wy + r;
        jw[r] = ((jr0 + y - 1) % jm + jm) % jm + 1;  // periodic j
        wrapn[r] = JODD && jw[r] == jm;
        wraps[r] = JODD && jw[r] == 1;
        coff[r] = IX(g, ir0, jw[r], 0) + kTbCW * lane;
        c3l[r] = g.cn3l[jw[r]];
        c3s[r] = g.cn3s[jw[r]];
        cB[r] = CN1K ? 0.0f : g.cnB[jw[r]];
        row0[r] = (y >= 1 && y < RH - 1);
        row1[r] = (y >= 2 && y < RH - 2);
        acc_cells[r] = (y >= 2 && y < 2 + ty && jr0 + y <= jm) && lane_tile;
        d0[r] = y * RW4 + lane;
    }
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
    // x parity of the colour-0 columns of each row at the first step
    const int par0 = (jw[0] + 1 - ir0 + kb) & 1, par1 = (jw[1] + 1 - ir0 + kb) & 1;

    auto request = [&](int k, int slot) {
        if (k <= ke) {
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const float *gsrc = pin + coff[r], *bsrc = a.rhs + coff[r];
                tb_cp_async16(reinterpret_cast<float *>(P + slot * RA4 + d0[r]), gsrc + pstride * k);
                tb_cp_async16(reinterpret_cast<float *>(Bs + slot * RA4 + d0[r]), bsrc + pstride * k);
                if (wrapn[r] || wraps[r])  // row jm -> side row 0, row 1 -> side row 1
                    tb_cp_async16(reinterpret_cast<float *>(Sd + (2 * slot + (wraps[r] ? 1 : 0)) * RW4 + lane),
                                  gsrc + pstride * k);
            }
        }
        tb_cp_commit();
    };
    // planes kb .. kb+D-1 in flight, then plane kb waited for
#pragma unroll
    for (int q = 0; q <= D; ++q) request(kb + q, q);
    tb_cp_wait<D>();
    __syncthreads();
    // windows w[r][x][c]: row r, column c of the plane whose step phase is x
    // (planes tau+1, tau, tau-1, tau-2 at phases m+1, m, m-1, m-2 of step m)
    float w[2][4][kTbCW];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const float4 v = P[d0[r]];  // plane kb, slot 0
        w[r][0][0] = v.x, w[r][0][1] = v.y, w[r][0][2] = v.z, w[r][0][3] = v.w;
#pragma unroll
        for (int c = 0; c < kTbCW; ++c) {
            w[r][3][c] = w[r][0][c];  // plane kb-1: the bottom ghost (kb = 1) or a ring plane
            w[r][1][c] = 0.0f;
            w[r][2][c] = 0.0f;
        }
    }
    unsigned long long fh = 0, flo = 0;
    int bad = 0;
    float fsum = 0.0f;
    float bk[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};  // per row: rhs of the colour-1 columns of the last colour-0 plane
    const int tau_end = k1 + 1;  // plane k1 is stored at this step
    // (DD: and tiles with columns outside the summed ones olo..ohi, whose sums test fl bit 3)
    const bool edge = ir0 <= 1 || ir0 + kTbRW - 1 >= im || (DD && (ir0 + RX < g.olo || ir0 + RX + TX - 1 > g.ohi));

    // Steps kb .. tau_end, four per group.  PAR: row 0's colour-0 x parity
    // at the group's first step; DIFF: row 1's parity differs from row 0's
    // (it does unless the rows meet across the boundary with odd jm); FAST:
    // FP32 residual; EDGE: i ghosts by select.
    auto run = [&](auto PARc, auto DIFFc, auto FASTc, auto EDGEc) {
        constexpr int PAR = decltype(PARc)::value, DIFF = decltype(DIFFc)::value;
        constexpr bool FAST = decltype(FASTc)::value, EDGE = decltype(EDGEc)::value;
        int slot1 = 1;  // slot of plane tau+1
        for (int tau0 = kb; tau0 <= tau_end; tau0 += 4) {
            auto step = [&](auto Mc) {
                constexpr int m = decltype(Mc)::value;
                constexpr int XN = (m + 1) & 3, XC = m & 3, XD = (m + 3) & 3, XDD = (m + 2) & 3;
                const int tau = tau0 + m;
                if (tau > tau_end) return;
                const int sq1 = slot1, sq0 = slot1 == 0 ? NS - 1 : slot1 - 1, sqm = sq0 == 0 ? NS - 1 : sq0 - 1;
                int sreq = slot1 + D;
                if (sreq >= NS) sreq -= NS;
                request(tau + 1 + D, sreq);
                tb_cp_wait<D>();
                __syncthreads();
                // incoming plane tau+1 (above ke: the top ghost, or a ring plane)
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    if (tau + 1 <= ke) {
                        const float4 v = P[sq1 * RA4 + d0[r]];
                        w[r][XN][0] = v.x, w[r][XN][1] = v.y, w[r][XN][2] = v.z, w[r][XN][3] = v.w;
                    } else {
#pragma unroll
                        for (int c = 0; c < kTbCW; ++c) w[r][XN][c] = w[r][XC][c];
                    }
                }
                auto upd = [&](int r, float &pc_ref, float west, float east, float pn, float ps, float pu, float pd,
                               float b, float c4l, float c4s, float cnq, float cC, int C, bool acc) {
                    const float pc = pc_ref;
                    const float pe = (EDGE && (fl[C] & 4)) ? pc : east;
                    const float pw = (EDGE && (fl[C] & 2)) ? pc : west;
                    const float cn1 = CN1K ? cnq : 1.0f / (cA[C] + cB[r] + cC);
                    const float reltmp = omega * (cn1 * (c2l[C] * pe + c2s[C] * pw + c3l[r] * pn + c3s[r] * ps +
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
                // the rhs kept by the previous step's colour 0 (plane tau-1), for
                // this step's colour 1, before this step's colour 0 replaces it
                float bkp[2][2];
#pragma unroll
                for (int r = 0; r < 2; ++r) bkp[r][0] = bk[r][0], bkp[r][1] = bk[r][1];
                // One half-sweep of row r on window phase X (plane pl, slot sq),
                // the k neighbours at phases XU (above) and XL (below); its
                // in-warp neighbour row's values from the copy o.
                auto half = [&](auto Rc, auto Xc, auto XUc, auto XLc, auto C0c, int pl, int sq, const float (&o)[kTbCW],
                                bool stores) {
                    constexpr int r = decltype(Rc)::value, X = decltype(Xc)::value;
                    constexpr int XU = decltype(XUc)::value, XL = decltype(XLc)::value, C0 = decltype(C0c)::value;
                    const float4 *Pq = P + sq * RA4 + d0[r];
                    float4 nn, ss;
                    if constexpr (r == 0) {  // row 1 of the warp above: row y+1 is row 1 of this warp
                        nn = make_float4(o[0], o[1], o[2], o[3]);
                        ss = wraps[0] ? Sd[2 * sq * RW4 + lane] : Pq[-RW4];
                    } else {
                        nn = wrapn[1] ? Sd[(2 * sq + 1) * RW4 + lane] : Pq[RW4];
                        ss = make_float4(o[0], o[1], o[2], o[3]);
                    }
                    // rhs: colour 0 loads the row's plane and keeps the other two
                    // columns for colour 1 on the same plane at the next step
                    float4 bb;
                    if (!stores) {
                        bb = Bs[sq * RA4 + d0[r]];
                        bk[r][0] = C0 == 0 ? bb.y : bb.x;
                        bk[r][1] = C0 == 0 ? bb.w : bb.z;
                    } else if constexpr (C0 == 0) {
                        bb = make_float4(bkp[r][0], 0.0f, bkp[r][1], 0.0f);
                    } else {
                        bb = make_float4(0.0f, bkp[r][0], 0.0f, bkp[r][1]);
                    }
                    const float c4l = kq.c4l[pl], c4s = kq.c4s[pl];
                    const float cnq = CN1K ? kq.cnk[pl] : 0.0f, cC = CN1K ? 0.0f : g.cnC[pl];
                    const bool acc = acc_cells[r] && pl >= k0 && pl <= k1;
                    float(&v)[kTbCW] = w[r][X];
                    if constexpr (C0 == 0) {
                        const float nb = __shfl_sync(0xffffffffu, v[3], lane - 1);
                        upd(r, v[0], nb, v[1], nn.x, ss.x, w[r][XU][0], w[r][XL][0], bb.x, c4l, c4s, cnq, cC, 0, acc);
                        upd(r, v[2], v[1], v[3], nn.z, ss.z, w[r][XU][2], w[r][XL][2], bb.z, c4l, c4s, cnq, cC, 2,
                            acc);
                    } else {
                        const float nb = __shfl_sync(0xffffffffu, v[0], lane + 1);
                        upd(r, v[1], v[0], v[2], nn.y, ss.y, w[r][XU][1], w[r][XL][1], bb.y, c4l, c4s, cnq, cC, 1,
                            acc);
                        upd(r, v[3], v[2], nb, nn.w, ss.w, w[r][XU][3], w[r][XL][3], bb.w, c4l, c4s, cnq, cC, 3, acc);
                    }
                    if (!stores) {
                        // colour 0: publish (the colour-1 columns are rewritten with the same bits)
                        P[sq * RA4 + d0[r]] = make_float4(v[0], v[1], v[2], v[3]);
                    } else if (acc) {
                        // colour 1: plane pl is final, store the tile part of the row
                        float *dst = pout + (coff[r] + pstride * pl);
                        if (!EDGE || (fl[3] & fl[0] & 1))
                            *reinterpret_cast<float4 *>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                        else {
#pragma unroll
                            for (int c = 0; c < kTbCW; ++c)
                                if (fl[c] & 1) dst[c] = v[c];
                        }
                    }
                };
                constexpr int CA = (PAR + m) & 1, CB = (PAR + DIFF + m) & 1;
                // colour 0 on plane tau; the in-warp neighbours as before the half-sweep
                if (tau <= ke) {
                    float o0[kTbCW], o1[kTbCW];
#pragma unroll
                    for (int c = 0; c < kTbCW; ++c) o0[c] = w[0][XC][c], o1[c] = w[1][XC][c];
                    if (row0[0]) half(IC<0>(), IC<XC>(), IC<XN>(), IC<XD>(), IC<CA>(), tau, sq0, o1, false);
                    if (row0[1]) half(IC<1>(), IC<XC>(), IC<XN>(), IC<XD>(), IC<CB>(), tau, sq0, o0, false);
                }
                // colour 1 on plane tau-1 (the same x parities as colour 0 on plane tau)
                const int q = tau - 1;
                if (q >= kb) {
                    float o0[kTbCW], o1[kTbCW];
#pragma unroll
                    for (int c = 0; c < kTbCW; ++c) o0[c] = w[0][XD][c], o1[c] = w[1][XD][c];
                    if (row1[0]) half(IC<0>(), IC<XD>(), IC<XC>(), IC<XDD>(), IC<CA>(), q, sqm, o1, true);
                    if (row1[1]) half(IC<1>(), IC<XD>(), IC<XC>(), IC<XDD>(), IC<CB>(), q, sqm, o0, true);
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
    const bool diff = par0 != par1;
#define S1P_RUN(F, E)                                      \
    do {                                                   \
        if (diff) {                                        \
            if (par0)                                      \
                run(IC<1>(), IC<1>(), F(), E());           \
            else                                           \
                run(IC<0>(), IC<1>(), F(), E());           \
        } else if (JODD) {                                 \
            if (par0)                                      \
                run(IC<1>(), IC<0>(), F(), E());           \
            else                                           \
                run(IC<0>(), IC<0>(), F(), E());           \
        }                                                  \
    } while (0)
    if (fast) {
        if (edge)
            S1P_RUN(True, True);
        else
            S1P_RUN(True, False);
    } else {
        if (edge)
            S1P_RUN(False, True);
        else
            S1P_RUN(False, False);
    }
#undef S1P_RUN
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
