// les_press.cuh -- pressure part of the time step (press.f95:49-146).
//
// Global sums use the exact fixed-point definition of les_fix.h: each
// reducing kernel writes one FixPart per block to a scratch array and a
// one-block kernel finishes the total.  The SOR loop runs on the device
// without host round trips: the residual kernel sets a converged flag and
// every later kernel of the loop returns at once when it is set.
#pragma once
#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

constexpr int kRedBX = 32, kRedBY = 8, kRedNT = kRedBX * kRedBY;
constexpr int kRedKMax = 8;  // planes per thread of the reduction grids (red_kchunk <= 8)

// bondFG.f95:15-31 fused with the rhs of press.f95:114-125 and the partial
// sums of press.f95:128-137.  rhs is stored before the rhsav subtraction
// (every reader subtracts the scalar itself).  Threads loop over a k chunk.
// 6 CTAs per SM (at most 42 registers): the loads of more warps in flight hide
// the memory latency that bounds this kernel
__global__ void __launch_bounds__(kRedNT, 6) k_rhs(Geo g, Fields F, int kchunk, FixPart *part) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    const bool own = i >= g.olo && i <= g.ohi;
    i128 acc = 0;
    int bad = 0;
    if (i <= g.im && j <= g.jm) {
        const float *dx1 = g.dx1, *dy1 = g.dy1, *dzn = g.dzn;
        // RN(1/dt) for kdiv; 0 (IEEE division) outside [2^-30, 2^30]
        const float rdt = (g.dt >= 0x1p-30f && g.dt <= 0x1p30f) ? 1.0f / g.dt : 0.0f;
        for (int k = k0; k <= k1; ++k) {
            // every load first (no store below writes a location any thread
            // reads), then the bondfg ghost writes, then rhs
            const int c = IX(g, i, j, k);
            const float fc = F.f[c], gc = F.g[c];
            float hc = F.h[c];
            const float fm = (i == 1) ? fc : F.f[IX(g, i - 1, j, k)];
            const float gm = (j == 1) ? F.g[IX(g, i, g.jm, k)] : F.g[IX(g, i, j - 1, k)];
            const float hm = (k == 1) ? 0.0f : F.h[IX(g, i, j, k - 1)];
            const float um = F.u[IX(g, i - 1, j, k)], uc = F.u[c];
            const float vm = F.v[IX(g, i, j - 1, k)], vc = F.v[c];
            const float wm = F.w[IX(g, i, j, k - 1)], wc = F.w[c];
            // bondfg: f(0,j,k)=f(1,j,k); g(i,0,k)=g(i,jm,k); h(i,j,0)=h(i,j,km)=0
            if (i == 1) F.f[IX(g, 0, j, k)] = fc;
            if (j == g.jm) F.g[IX(g, i, 0, k)] = gc;
            if (k == g.km) {
                F.h[c] = 0.0f;
                hc = 0.0f;
            }
            if (k == 1) F.h[IX(g, i, j, 0)] = 0.0f;
            // the quotients of press.f95:59-70 with the IEEE bits: by an x/y
            // spacing, a multiplication when its reciprocal is an exact power
            // of two (fdiv); by dzn(k) and dt, Markstein's corrected quotient
            // from the rounded reciprocal (kdiv)
            const float rdx = g.rdx1[i], rdy = g.rdy1[j], dz = dzn[k], rdz = g.rdzn[k];
            float r = fdiv(-um + uc, dx1[i], rdx) + fdiv(-vm + vc, dy1[j], rdy) + kdiv(-wm + wc, dz, rdz);
            r = fdiv(fc - fm, dx1[i], rdx) + fdiv(gc - gm, dy1[j], rdy) + kdiv(hc - hm, dz, rdz) + kdiv(r, g.dt, rdt);
            F.rhs[c] = r;
            if (own) acc += fix_term(dx1[i] * dy1[j] * dzn[k] * r, bad);
        }
    }
    block_fix_sum<kRedNT>(acc, bad, &part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)]);
}

// Sum FixParts part[b*stride + off], b < n, with one block; thread 0 gets
// the total.  Ends with the block synchronised.
__device__ __forceinline__ void final_fix_strided(const FixPart *part, int n, int stride, int off, i128 &tot,
                                                  int &bad) {
    __shared__ unsigned long long s_lo[32];
    __shared__ long long s_hi[32];
    __shared__ int s_bad[32];
    i128 acc = 0;
    int b = 0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const FixPart &q = part[(size_t)t * stride + off];
        acc += fix_from_part(q);
        b |= q.bad;
    }
    for (int o = 16; o >= 1; o >>= 1) {
        acc += shfl_down_i128(acc, o);
        b |= __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_lo[wid] = (unsigned long long)acc;
        s_hi[wid] = (long long)(acc >> 64);
        s_bad[wid] = b;
    }
    __syncthreads();
    tot = 0;
    bad = 0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            tot += (i128)(((unsigned __int128)(unsigned long long)s_hi[w] << 64) | (unsigned __int128)s_lo[w]);
            bad |= s_bad[w];
        }
    }
    __syncthreads();
}

// Sum FixParts with one block; the finisher maps the total to the scalars.
__device__ __forceinline__ void final_fix(const FixPart *part, int n, i128 &tot, int &bad) {
    __shared__ unsigned long long s_lo[32];
    __shared__ long long s_hi[32];
    __shared__ int s_bad[32];
    i128 acc = 0;
    int b = 0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        acc += fix_from_part(part[t]);
        b |= part[t].bad;
    }
    for (int off = 16; off >= 1; off >>= 1) {
        acc += shfl_down_i128(acc, off);
        b |= __shfl_down_sync(0xffffffffu, b, off);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_lo[wid] = (unsigned long long)acc;
        s_hi[wid] = (long long)(acc >> 64);
        s_bad[wid] = b;
    }
    __syncthreads();
    tot = 0;
    bad = 0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            tot += (i128)(((unsigned __int128)(unsigned long long)s_hi[w] << 64) | (unsigned __int128)s_lo[w]);
            bad |= s_bad[w];
        }
    }
}

// Exact sum (Q63.64 terms, les_fix.h) of a field over its Fortran bounds,
// one partial per block (kRedNT threads); rhs as the caller sees it
// (rhs - rhsav on the interior when sub_interior).
__global__ void __launch_bounds__(kRedNT) k_field_sum(Geo g, const float *__restrict__ box, int li, int lj, int lk,
                                                      int ni, int nj, int nk, const Scal *s, int sub_interior,
                                                      FixPart *part) {
    const size_t n = (size_t)ni * nj * nk;
    const float sub = sub_interior ? s->rhsav : 0.0f;
    i128 acc = 0;
    int bad = 0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int i = li + (int)(t % ni), r = (int)(t / ni);
        const int j = lj + r % nj, k = lk + r / nj;
        float x = box[IX(g, i, j, k)];
        if (sub_interior && i >= 1 && i <= g.im && j >= 1 && j <= g.jm && k >= 1 && k <= g.km) x = x - sub;
        acc += fix_term(x, bad);
    }
    block_fix_sum<kRedNT>(acc, bad, &part[blockIdx.x]);
}

__global__ void __launch_bounds__(1024) k_field_sum_final(const FixPart *part, int n, double *out) {
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
    if (threadIdx.x == 0) *out = fix_finish(tot, bad);
}

// rhsav = num/area (press.f95:138), area given (grid-only, finished on the host).
__global__ void __launch_bounds__(1024) k_final_rhsav(const FixPart *part, int n, double area, Scal *s) {
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
    if (threadIdx.x == 0) s->rhsav = (float)(fix_finish(tot, bad) / area);
}

// One SOR colour sweep, press.f95:153-163 with nrd = colour: cells with
// (i+j+k+nrd) odd.  Within a colour every update reads only cells of the
// other colour and ghost cells, so the in-place parallel sweep equals the
// reference's sequential one.  cn1 is rebuilt from its separable parts, or
// read from the caller's array (CN1MEM, the per-routine press entry).
// r2 (may be NULL): each swept cell's reltmp^2 stored at its box index, for
// the reference-order residual sum (k_seq_sum).
template <bool CN1MEM>
__global__ void __launch_bounds__(kRedNT) k_sor_colour(Geo g, float *__restrict__ p, const float *__restrict__ rhs,
                                                        const float *__restrict__ cn1b, int nrd, int kchunk,
                                                        FixPart *part, const Scal *s, float *__restrict__ r2) {
    if (s->converged) return;
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    const float rhsav = s->rhsav;
    const bool own = i >= g.olo && i <= g.ohi;
    i128 acc = 0;
    int bad = 0;
    if (i <= g.im && j <= g.jm) {
        const float cA = g.cnA[i], c2l = g.cn2l[i], c2s = g.cn2s[i];
        const float cB = g.cnB[j], c3l = g.cn3l[j], c3s = g.cn3s[j];
        int k = k0 + (((i + j + k0 + nrd) & 1) ? 0 : 1);
        for (; k <= k1; k += 2) {
            const int c = IX(g, i, j, k);
            const float cn1 = CN1MEM ? cn1b[c] : 1.0f / (cA + cB + g.cnC[k]);
            const float pc = p[c];
            const float reltmp =
                g.omega * (cn1 * (c2l * p[c + 1] + c2s * p[c - 1] + c3l * p[c + g.si] + c3s * p[c - g.si] +
                                  g.cn4l[k] * p[c + g.si * g.sj] + g.cn4s[k] * p[c - g.si * g.sj] -
                                  (rhs[c] - rhsav)) -
                           pc);
            p[c] = pc + reltmp;
            if (own) acc += fix_term(reltmp * reltmp, bad);
            if (r2) r2[c] = reltmp * reltmp;
        }
    }
    block_fix_sum<kRedNT>(acc, bad, &part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)]);
}

// boundp.f95:23-44 (boundp1) as final values: ghost (i,j,k), k in 0..km+1,
// = p(ci, pj, k) with ci clamping i to 1..im and pj the periodic j map.
// CHECK=true: part of the SOR loop (skipped once converged).
template <bool CHECK>
__global__ void __launch_bounds__(256) k_boundp1(Geo g, float *__restrict__ p, const Scal *s) {
    if (CHECK && s->converged) return;
    const int im = g.im, jm = g.jm, km = g.km;
    const int nI = 2 * (jm + 2) * (km + 2);  // i=0,im+1 ; j=0..jm+1
    const int nJ = 2 * im * (km + 2);        // j=0,jm+1 ; i=1..im
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t < nI) {
        i = (t & 1) ? im + 1 : 0;
        const int r = t >> 1;
        j = r % (jm + 2);
        k = r / (jm + 2);
    } else if ((t -= nI) < nJ) {
        j = (t & 1) ? jm + 1 : 0;
        const int r = t >> 1;
        i = 1 + r % im;
        k = r / im;
    } else {
        return;
    }
    const int ci = i < 1 ? 1 : (i > im ? im : i);
    const int pj = (j == 0) ? jm : (j == jm + 1 ? 1 : j);
    p[IX(g, i, j, k)] = p[IX(g, ci, pj, k)];
}

// boundp.f95:5-21 (boundp2): p(i,j,0)=p(i,j,1), p(i,j,km+1)=p(i,j,km).
template <bool CHECK>
__global__ void __launch_bounds__(256) k_boundp2(Geo g, float *__restrict__ p, const Scal *s) {
    if (CHECK && s->converged) return;
    const int ni = g.im + 2, nj = g.jm + 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * ni * nj) return;
    const int i = t % ni, r = t / ni;
    const int j = r % nj;
    const bool top = (r / nj) != 0;
    if (top)
        p[IX(g, i, j, g.km + 1)] = p[IX(g, i, j, g.km)];
    else
        p[IX(g, i, j, 0)] = p[IX(g, i, j, 1)];
}

// press.f95:114: after iteration l, stop when sor < pjuge.
__global__ void __launch_bounds__(1024) k_final_sor(const FixPart *part, int n, float pjuge, Scal *s) {
    if (s->converged) return;
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
    if (threadIdx.x == 0) {
        const float sor = (float)fix_finish(tot, bad);
        s->sor = sor;
        s->sor_iters += 1;
        if (sor < pjuge) s->converged = 1;
    }
}

// press.f95:186-195 partial sums of p*dx1*dy1*dzn.
__global__ void __launch_bounds__(kRedNT) k_pav_reduce(Geo g, const float *p0, const float *p1, int kchunk,
                                                        FixPart *part, const Scal *sc) {
    const float *__restrict__ p = sc->pbuf ? p1 : p0;
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    const bool own = i >= g.olo && i <= g.ohi;
    i128 acc = 0;
    int bad = 0;
    if (i <= g.im && j <= g.jm) {
        // the chunk's loads first (kchunk <= kRedKMax), then the sums
        float pv[kRedKMax];
#pragma unroll
        for (int q = 0; q < kRedKMax; ++q) pv[q] = (k0 + q <= k1) ? p[IX(g, i, j, k0 + q)] : 0.0f;
#pragma unroll
        for (int q = 0; q < kRedKMax; ++q)
            if (own && k0 + q <= k1) acc += fix_term(pv[q] * g.dx1[i] * g.dy1[j] * g.dzn[k0 + q], bad);
    }
    block_fix_sum<kRedNT>(acc, bad, &part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)]);
}

__global__ void __launch_bounds__(1024) k_final_pav(const FixPart *part, int n, double area, Scal *s) {
    i128 tot;
    int bad;
    final_fix(part, n, tot, bad);
    if (threadIdx.x == 0) s->pav = (float)(fix_finish(tot, bad) / area);
}

// press.f95:197-209: p -= pav on the interior, then boundp1 and boundp2.
// The interior thread writes its new value and every ghost whose final
// source it is: ghost (i,j,k) <- (clamp(i), periodic(j), clamp(k)).  The
// SOR result may sit in the second buffer (s->pbuf); the state p is written.
__global__ void __launch_bounds__(kRedNT) k_pav_adjust(Geo g, float *p, const float *p1, const Scal *s, int kchunk) {
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.km, k0 + kchunk - 1);
    if (i > g.im || j > g.jm) return;
    const float *src = s->pbuf ? p1 : p;
    const float pav = s->pav;
    // the chunk's loads first (kchunk <= kRedKMax): the stores below write
    // this thread's own cells and ghosts only, which no thread reads here
    float pv[kRedKMax];
#pragma unroll
    for (int q = 0; q < kRedKMax; ++q) pv[q] = (k0 + q <= k1) ? src[IX(g, i, j, k0 + q)] : 0.0f;
#pragma unroll
    for (int q = 0; q < kRedKMax; ++q) {
        const int k = k0 + q;
        if (k > k1) break;
        const float val = pv[q] - pav;
        // the cell and its boundp1/boundp2 copies: at most one extra i, j and k
        // (im, jm >= 2, km >= 3)
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
}

// ---------------------------------------------------------------------------
// Reference-order sums (reduction mode bits LES_RED_F_*): the sequential FP32
// loops of press.f95 restated exactly, for parity runs against the
// reference's own summation order.
//   kind 0: rhsav = sum(dx1*dy1*dzn*rhs) / sum(dx1*dy1*dzn), press.f95:66-75
//   kind 1: sor = sum(reltmp^2) over colour 0 then colour 1, each in
//           (k, j, i) order, press.f95:87-99, and the stop test of :114
//   kind 2: pav = sum(p*dx1*dy1*dzn) / sum(dx1*dy1*dzn), press.f95:123-133
// A serial FP32 sum has one order, so one block does it: the threads walk
// the interior in Fortran order in chunks of kSeqChunk cells, each thread
// loads kSeqPer cells of the chunk, the terms that take part are packed in
// order into shared memory (warp ballots plus a prefix over the warps), and
// thread 0 adds them one after another.  A test mode: about 4 cycles per
// term, so milliseconds per sum at 2 M cells.
constexpr int kSeqNT = 512, kSeqPer = 8, kSeqChunk = kSeqNT * kSeqPer;

template <int KIND>
__global__ void __launch_bounds__(kSeqNT, 1) k_seq_sum(Geo g, const float *__restrict__ a0,
                                                        const float *__restrict__ a1, float pjuge, Scal *s) {
    __shared__ float ta[kSeqChunk];
    __shared__ float tb[KIND == 1 ? 1 : kSeqChunk];
    __shared__ int wcount[kSeqNT / 32];
    if (KIND == 1 && s->converged) return;
    const float *__restrict__ src = (KIND == 2 && s->pbuf) ? a1 : a0;
    const int N = g.im * g.jm * g.km;  // < 2^31: the padded box is (les_ctx_create)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float acc = 0.0f, acc2 = 0.0f;  // thread 0's running sums
    for (int colour = 0; colour < (KIND == 1 ? 2 : 1); ++colour) {
        for (int base = 0; base < N; base += kSeqChunk) {
            float x[kSeqPer], y[kSeqPer];
            bool take[kSeqPer];
#pragma unroll
            for (int q = 0; q < kSeqPer; ++q) {
                const int t = base + q * kSeqNT + (int)threadIdx.x;
                take[q] = false;
                x[q] = 0.0f;
                y[q] = 0.0f;
                if (t < N) {
                    const int r = t / g.im, i = 1 + (t - r * g.im);
                    const int k = 1 + r / g.jm, j = 1 + (r - (k - 1) * g.jm);
                    const int c = IX(g, i, j, k);
                    if (KIND == 1) {
                        // colour nrd: i = 1 + mod(k+j+nrd, 2), step 2, i.e. i+j+k+nrd odd
                        take[q] = ((i + j + k + colour) & 1) != 0;
                        if (take[q]) x[q] = src[c];
                    } else if (KIND == 0) {
                        const float w = g.dx1[i] * g.dy1[j] * g.dzn[k];
                        x[q] = w * src[c];
                        y[q] = w;
                        take[q] = true;
                    } else {
                        x[q] = src[c] * g.dx1[i] * g.dy1[j] * g.dzn[k];
                        y[q] = g.dx1[i] * g.dy1[j] * g.dzn[k];
                        take[q] = true;
                    }
                }
            }
            int packed = 0;  // terms of this chunk packed so far
#pragma unroll
            for (int q = 0; q < kSeqPer; ++q) {
                const unsigned m = __ballot_sync(0xffffffffu, take[q]);
                if (lane == 0) wcount[wid] = __popc(m);
                __syncthreads();
                int off = packed, total = packed;
                for (int w = 0; w < kSeqNT / 32; ++w) {
                    const int cw = wcount[w];
                    if (w < wid) off += cw;
                    total += cw;
                }
                if (take[q]) {
                    const int pos = off + __popc(m & ((1u << lane) - 1u));
                    ta[pos] = x[q];
                    if (KIND != 1) tb[pos] = y[q];
                }
                packed = total;
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                if (KIND == 1) {
                    for (int t = 0; t < packed; ++t) acc = acc + ta[t];
                } else {
                    for (int t = 0; t < packed; ++t) {
                        acc = acc + ta[t];
                        acc2 = acc2 + tb[t];
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;
    if (KIND == 0) {
        s->rhsav = acc / acc2;
    } else if (KIND == 1) {
        s->sor = acc;
        s->sor_iters += 1;
        if (acc < pjuge) s->converged = 1;
    } else {
        s->pav = acc / acc2;
    }
}

// Per-step scalars reset and the centre probe of press.f95:183-187.
__global__ void k_step_begin(Scal *s, int n) {
    s->uout_pos = 0u;
    s->uout_neg = 0u;
    s->converged = 0;
    s->sor_iters = 0;
    s->redo = 0;
    s->pbuf = 0;
    s->exact_sums = 0;
    s->n = n;
}
// k_step_begin with n read from device memory (ensemble graphs: one
// captured graph serves every step, k_ens_advance moves n on).
__global__ void k_step_begin_dev(Scal *s, const int *n) {
    s->uout_pos = 0u;
    s->uout_neg = 0u;
    s->converged = 0;
    s->sor_iters = 0;
    s->redo = 0;
    s->pbuf = 0;
    s->exact_sums = 0;
    s->n = *n;
}
__global__ void k_ens_advance(int *n) { *n += 1; }
__global__ void k_probe(Geo g, Fields F, Scal *s) {
    const int c = IX(g, g.im / 2, g.jm / 2, g.km / 2);
    s->probe[0] = F.p[c];
    s->probe[1] = F.u[c];
    s->probe[2] = F.v[c];
    s->probe[3] = F.w[c];
}

}  // namespace
}  // namespace les
