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
//   - the CTA owns a (64 - 4T) x ty tile of (i,j) columns and keeps a ring
//     of R = 2*T cells around it (each region row is 64 floats); half-sweep s
//     updates the ring shrunk to width R-s-1, so after 2T half-sweeps the
//     tile holds exact values;
//   - planes march k = 1..km: at step tau half-sweep s works on plane
//     tau-s, in order s = 0,1,.., so each plane sees its neighbours at the
//     right level;
//   - each region row is stored parity-split (even x, then odd x): a colour
//     sweep and its x+-1 neighbours are unit-stride across the lanes of a
//     warp, free of bank conflicts;
//   - a warp owns whole rows, a lane one cell of the row's colour;
//   - planes are staged with cp.async several steps ahead of their use;
//   - p is read from one buffer and written to the other (nothing a
//     neighbouring CTA reads is overwritten);
//   - reltmp^2 of the tile cells is summed per iteration (les_fix.h).
// A pass that converges part-way (sor < pjuge before its last iteration) is
// redone from its input buffer with exactly the iterations the reference
// executes.
#pragma once
#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

constexpr int kTbRW = 64, kTbNW = 8, kTbNT = 32 * kTbNW;
constexpr int kTbTMax = 3;
constexpr int kTbDepth = 3;   // planes in flight ahead of the one a step needs
constexpr int kTbMaxRH = 64;  // region rows (tile rows + 2 rings)

__host__ __device__ constexpr int tb_ring(int T) { return 2 * T; }
// tile columns: the 64-column region minus a ring on each side
__host__ __device__ constexpr int tb_tx(int T) { return kTbRW - 2 * tb_ring(T); }
// shared memory plane slots (see the pipeline notes in k_sor_tb)
__host__ __device__ constexpr int tb_np(int T) { return kTbDepth + 2 * T + 2; }
__host__ __device__ constexpr int tb_nb(int T) { return kTbDepth + 2 * T; }
__host__ __device__ inline int tb_rh(int T, int ty) { return ty + 2 * tb_ring(T); }
// plane slots plus the per-row tables (cn3l, cn3s, cnB, box offset)
__host__ __device__ inline size_t tb_smem(int T, int ty) {
    return sizeof(float) * ((size_t)kTbRW * tb_rh(T, ty) * (tb_np(T) + tb_nb(T)) + 4 * kTbMaxRH);
}
__host__ __device__ inline bool tb_fits(int T, int ty) { return ty >= 1 && tb_rh(T, ty) <= kTbMaxRH; }

// Exact Q63.64 term for a non-negative float below 2^62 (les_fix.h): the
// integer part and the fraction scaled by 2^64, both exact in FP64.
__device__ __forceinline__ void fix_add_nonneg(float x, unsigned long long &hi, unsigned long long &lo, int &bad) {
    if (!(x < 4.611686018427388e18f)) {  // NaN, inf or >= 2^62
        bad = 1;
        return;
    }
    const double d = (double)x;
    const double ip = floor(d);
    const unsigned long long fr = __double2ull_rz((d - ip) * 18446744073709551616.0);
    const unsigned long long o = lo;
    lo += fr;
    hi += (unsigned long long)ip + (lo < o ? 1ull : 0ull);
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

// One pass of T iterations (mode 0) or of scal->redo iterations (mode 1,
// recomputing a pass that converged part-way; niter is then ignored).
// CN1K: cn1 depends on k only (uniform dx and dy), read from cn1k[k].
//
// Pipeline: step tau works on planes tau - 2*nit + 1 .. tau and needs p of
// planes tau - 2*nit .. tau + 1 and rhs of the planes it updates.  Plane
// tau + kTbDepth is requested (cp.async, one group per plane) at the start
// of step tau into the slot of plane tau + kTbDepth - NP, which no thread
// has touched since step tau - 1; the wait then lets kTbDepth - 1 groups
// stay in flight.  A lane copies columns lane and lane + 32 of a row
// (128-byte coalesced reads) to their parity-split positions.  rhs is
// staged raw and rhsav subtracted where it is read (the same FP32
// subtraction the reference does once per cell).
template <int T, bool CN1K>
__global__ void __launch_bounds__(kTbNT) k_sor_tb(Geo g, float *pb0, float *pb1, const float *__restrict__ rhs,
                                                   const float *__restrict__ cn1k, int ty, int niter, int mode,
                                                   FixPart *part, Scal *sc) {
    extern __shared__ float smem[];
    if (mode == 0 && sc->converged) return;
    const int nit = (mode == 0) ? niter : sc->redo;
    if (nit <= 0) return;
    constexpr int R = tb_ring(T), NP = tb_np(T), NB = tb_nb(T), D = kTbDepth;
    const int nhs = 2 * nit;
    const int RH = tb_rh(T, ty), RA = kTbRW * RH;
    float *P = smem;
    float *B = P + NP * RA;
    float *s_c3l = B + NB * RA, *s_c3s = s_c3l + kTbMaxRH, *s_cB = s_c3s + kTbMaxRH;
    int *s_goff = reinterpret_cast<int *>(s_cB + kTbMaxRH);  // box offset of (ir0, j, k = 0)
    const float *pin = sc->pbuf ? pb1 : pb0;
    float *pout = sc->pbuf ? pb0 : pb1;
    const float rhsav = sc->rhsav, omega = g.omega;
    const int im = g.im, jm = g.jm, km = g.km;
    constexpr int TX = tb_tx(T);
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * ty;
    const int ir0 = i0 - R, jr0 = j0 - R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long pstride = (long long)g.si * g.sj;

    for (int y = threadIdx.x; y < RH; y += kTbNT) {
        const int jw = ((jr0 + y - 1) % jm + jm) % jm + 1;
        s_c3l[y] = g.cn3l[jw];
        s_c3s[y] = g.cn3s[jw];
        s_cB[y] = CN1K ? 0.0f : g.cnB[jw];
        s_goff[y] = IX(g, ir0, jw, 0);
    }
    // this lane's column of each parity: region x = par + 2*lane (scalars, not
    // arrays, so a run-time parity selects registers instead of local memory)
    float c2l0, c2l1, c2s0, c2s1, cA0, cA1;
    int fl0, fl1;  // bit 0: 1 <= i <= im, 1: i == 1, 2: i == im, 3: x inside the tile
    {
        auto col = [&](int par, float &cl, float &cs, float &ca, int &fl) {
            const int x = par + 2 * lane, i = ir0 + x;
            const bool ok = (i >= 1 && i <= im);
            cl = ok ? g.cn2l[i] : 0.0f;
            cs = ok ? g.cn2s[i] : 0.0f;
            ca = (!CN1K && ok) ? g.cnA[i] : 0.0f;
            fl = (ok ? 1 : 0) | (i == 1 ? 2 : 0) | (i == im ? 4 : 0) | ((x >= R && x < R + TX) ? 8 : 0);
        };
        col(0, c2l0, c2s0, cA0, fl0);
        col(1, c2l1, c2s1, cA1, fl1);
    }
    // reltmp^2 sums of the pass's iterations 0, 1, 2 (named scalars: an
    // array indexed by the run-time iteration would live in local memory)
    unsigned long long h0 = 0, l0 = 0, h1 = 0, l1 = 0, h2 = 0, l2 = 0;
    int bad = 0;
    __syncthreads();

    // columns lane, lane+32 of region row y -> parity-split positions
    const int dA = (lane & 1) * 32 + (lane >> 1), dB = dA + 16;
    auto request = [&](int k) {
        if (k <= km) {
            float *Pp = P + (k % NP) * RA;
            float *Bp = B + (k % NB) * RA;
            const long long ko = pstride * k;
            for (int y = warp; y < RH; y += kTbNW) {
                const long long src = s_goff[y] + ko + lane;
                tb_cp_async4(Pp + y * kTbRW + dA, pin + src);
                tb_cp_async4(Pp + y * kTbRW + dB, pin + src + 32);
                tb_cp_async4(Bp + y * kTbRW + dA, rhs + src);
                tb_cp_async4(Bp + y * kTbRW + dB, rhs + src + 32);
            }
        }
        tb_cp_commit();
    };

#pragma unroll
    for (int k = 1; k <= D; ++k) request(k);
    const int nsteps = km + nhs - 1;
    for (int tau = 1; tau <= nsteps; ++tau) {
        request(tau + D);
        tb_cp_wait<D - 1>();
        __syncthreads();
        for (int s = 0; s < nhs; ++s) {
            const int q = tau - s;
            if (q >= 1 && q <= km) {
                const int nrd = s & 1;
                const int lo = s + 1, hi_x = kTbRW - lo, hi_y = RH - lo;  // region R_{s+1}: [lo,hi)
                float *Pc = P + (q % NP) * RA;
                const float *Pu = P + ((q + 1) % NP) * RA;
                const float *Pd = P + ((q - 1 + NP) % NP) * RA;
                const float *Bc = B + (q % NB) * RA;
                const float c4l = g.cn4l[q], c4s = g.cn4s[q];
                const float cnq = CN1K ? cn1k[q] : 0.0f;
                const float cC = CN1K ? 0.0f : g.cnC[q];
                const bool top = (q == km), bottom = (q == 1);
                const int pb = (jr0 + q + nrd + 1 - ir0) & 1;  // x parity of the colour on row 0
                for (int yy = lo + warp; yy < hi_y; yy += kTbNW) {
                    const int par = (yy + pb) & 1;
                    const int x = par + 2 * lane;
                    const int fl = par ? fl1 : fl0;
                    if (x < lo || x >= hi_x || !(fl & 1)) continue;
                    const int o = yy * kTbRW + par * 32 + lane;
                    const int oe = yy * kTbRW + (1 - par) * 32 + lane + par;
                    const float pc = Pc[o];
                    const float pe = (fl & 4) ? pc : Pc[oe];
                    const float pw = (fl & 2) ? pc : Pc[oe - 1];
                    const float pn = Pc[o + kTbRW];
                    const float ps = Pc[o - kTbRW];
                    const float pu = top ? pc : Pu[o];
                    const float pd = bottom ? pc : Pd[o];
                    const float cn1 = CN1K ? cnq : 1.0f / ((par ? cA1 : cA0) + s_cB[yy] + cC);
                    const float reltmp =
                        omega * (cn1 * ((par ? c2l1 : c2l0) * pe + (par ? c2s1 : c2s0) * pw + s_c3l[yy] * pn +
                                        s_c3s[yy] * ps + c4l * pu + c4s * pd - (Bc[o] - rhsav)) -
                                 pc);
                    Pc[o] = pc + reltmp;
                    if (mode == 0 && (fl & 8) && yy >= R && yy < R + ty && jr0 + yy <= jm) {
                        const int t = s >> 1;
                        if (t == 0)
                            fix_add_nonneg(reltmp * reltmp, h0, l0, bad);
                        else if (T > 1 && t == 1)
                            fix_add_nonneg(reltmp * reltmp, h1, l1, bad);
                        else if (T > 2)
                            fix_add_nonneg(reltmp * reltmp, h2, l2, bad);
                    }
                }
            }
            __syncthreads();
        }
        const int qs = tau - nhs + 1;
        if (qs >= 1 && qs <= km) {
            const float *Ps = P + (qs % NP) * RA;
            const long long ko = pstride * qs;
            for (int yy = R + warp; yy < R + ty; yy += kTbNW) {
                if (jr0 + yy > jm) break;
                const float *row = Ps + yy * kTbRW;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int x = R + lane + 32 * h;  // tile columns R .. R+TX-1
                    if (x < R + TX && ir0 + x <= im) pout[s_goff[yy] + ko + x] = row[(x & 1) * 32 + (x >> 1)];
                }
            }
        }
    }
    tb_cp_wait<0>();  // nothing is in flight at exit (the last groups are empty)
    if (mode == 0) {
        const int b = blockIdx.x + gridDim.x * blockIdx.y;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            __syncthreads();
            const unsigned long long hi = t == 0 ? h0 : (t == 1 ? h1 : h2), lo = t == 0 ? l0 : (t == 1 ? l1 : l2);
            const i128 v = (i128)(((unsigned __int128)hi << 64) | (unsigned __int128)lo);
            block_fix_sum<kTbNT>(v, bad, &part[b * kTbTMax + t]);
        }
    }
}

// After a pass of niter iterations: the residual of each iteration in order
// (press.f95:114); stop at the first below pjuge.  A pass that stopped
// before its last iteration is marked for a redo of that many iterations.
__global__ void __launch_bounds__(1024) k_final_tb(const FixPart *part, int nblocks, int niter, float pjuge, Scal *s) {
    if (s->converged) return;
    __shared__ int stop;
    for (int t = 0; t < niter; ++t) {
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
                if (t < niter - 1) s->redo = t + 1;
                stop = 1;
            }
        }
        __syncthreads();
        if (stop) break;
    }
    if (threadIdx.x == 0 && s->redo == 0) s->pbuf ^= 1;
}

// After the redo kernel: the redone pass is the result.
__global__ void k_finish_redo(Scal *s) {
    if (s->redo) {
        s->redo = 0;
        s->pbuf ^= 1;
    }
}

}  // namespace
}  // namespace les
