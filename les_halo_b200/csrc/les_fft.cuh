// les_fft.cuh -- batched FP64 FFTs of contiguous lines for the spectral solve
// of the refined press (les_spectral.cuh): real-to-complex forward (the
// first n/2 + 1 coefficients) and complex-to-real inverse (unnormalised,
// the input taken as the half spectrum of a real line).
//
// Two real lines share one complex FFT: z = a + i b, Z = FFT z, then
// A_m = (Z_m + conj Z_{n-m}) / 2 and B_m = (Z_m - conj Z_{n-m}) / 2i; the
// inverse builds Z = A + i B from the two half spectra and takes a and b as
// the real and imaginary parts of its inverse FFT.  Line lengths are even
// and at most kFftPoints, line counts even.
//
// Mixed-radix Stockham autosort FFT in shared memory (radices 4, 5, 3, 2,
// 7, 11, 13, largest stages first): a stage of radix R with Ns points
// already combined reads v_r = a[j + r n/R] times the twiddle
// w^(r (j mod Ns) n/(Ns R)), w = exp(-2 pi i / n), takes their length-R DFT
// and writes it to a[(j div Ns) Ns R + (j mod Ns) + r Ns]; after the last
// stage the line is in natural order.  Two buffers in shared memory, one
// barrier per stage.  The twiddles come from host-built per-stage tables laid out
// so that a warp's butterflies read consecutive entries.  Radix 2, 3, 4, 5
// butterflies are written out with the roots' exact values; 7, 11 and 13
// take their roots from the table exp(-2 pi i k / n), k < n.  Products use
// fused multiply-adds.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

#include "les_dev.cuh"

namespace les {
namespace {

constexpr int kFftMaxStages = 24, kFftMaxRadix = 13, kFftThreads = 256, kFftPoints = 2048;
constexpr int kLoadBatch = 8;  // global loads of a thread issued together

struct FftPlan {
    int n, nstage;
    int radix[kFftMaxStages];
    int tofs[kFftMaxStages];  // stage s's twiddles at tw + tofs[s]: entry (r - 1) Ns + k
    const double2 *tw;        // per-stage twiddles, then exp(-2 pi i k / n), k = 0..n-1 (at tw + troot)
    int troot;
    int lpb;     // complex lines (pairs of real lines) per block and group
    int blocks;  // grid size cap (blocks loop over the groups)
};

// q div d and q mod d for 0 <= q < 2^20 and d >= 1 through a float
// reciprocal, corrected to the exact quotient.
__device__ __forceinline__ int fdiv_small(int q, int d, float rd) {
    int t = __float2int_rz((float)q * rd);
    if (t * d > q) --t;
    else if ((t + 1) * d <= q) ++t;
    return t;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// cos and sin of 2 pi / 5, 4 pi / 5 and sqrt(3) / 2.
constexpr double kC51 = 0.30901699437494742410, kC52 = -0.80901699437494742410;
constexpr double kS51 = 0.95105651629515357212, kS52 = 0.58778525229247312917;
constexpr double kS3 = 0.86602540378443864676;

// Length-R DFT of v in place, R = 2, 3, 4, 5: V_q = sum_r v_r exp(-2 pi i r q / R).
template <int R>
__device__ __forceinline__ void small_dft(double2 (&v)[R]) {
    if constexpr (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const double2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const double2 t = make_double2(fma(-0.5, s.x, v[0].x), fma(-0.5, s.y, v[0].y));
        v[0] = cadd(v[0], s);
        v[1] = make_double2(fma(kS3, d.y, t.x), fma(-kS3, d.x, t.y));  // t - i (sqrt3/2) d
        v[2] = make_double2(fma(-kS3, d.y, t.x), fma(kS3, d.x, t.y));
    } else if constexpr (R == 4) {  // roots 1, -i, -1, i
        const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const double2 s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = make_double2(d02.x + d13.y, d02.y - d13.x);  // d02 - i d13
        v[3] = make_double2(d02.x - d13.y, d02.y + d13.x);  // d02 + i d13
    } else if constexpr (R == 5) {
        // s1 = v1 + v4, d1 = v1 - v4, s2 = v2 + v3, d2 = v2 - v3:
        // V1,4 = v0 + c1 s1 + c2 s2 -+ i (s1' d1 + s2' d2)
        // V2,3 = v0 + c2 s1 + c1 s2 -+ i (s2' d1 - s1' d2)
        const double2 s1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
        const double2 s2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
        const double2 a1 = make_double2(fma(kC51, s1.x, fma(kC52, s2.x, v[0].x)),
                                        fma(kC51, s1.y, fma(kC52, s2.y, v[0].y)));
        const double2 a2 = make_double2(fma(kC52, s1.x, fma(kC51, s2.x, v[0].x)),
                                        fma(kC52, s1.y, fma(kC51, s2.y, v[0].y)));
        const double2 b1 = make_double2(fma(kS51, d1.x, kS52 * d2.x), fma(kS51, d1.y, kS52 * d2.y));
        const double2 b2 = make_double2(fma(kS52, d1.x, -(kS51 * d2.x)), fma(kS52, d1.y, -(kS51 * d2.y)));
        v[0] = cadd(v[0], cadd(s1, s2));
        v[1] = make_double2(a1.x + b1.y, a1.y - b1.x);  // a1 - i b1
        v[4] = make_double2(a1.x - b1.y, a1.y + b1.x);
        v[2] = make_double2(a2.x + b2.y, a2.y - b2.x);
        v[3] = make_double2(a2.x - b2.y, a2.y + b2.x);
    }
}

// Roots w_R^e = exp(-2 pi i e / R) of the composite radices 6, 8, 10 as
// exact constants (cos and sin of multiples of 60, 45 and 36 degrees).
constexpr double kS2 = 0.70710678118654752440;  // sqrt(2) / 2
template <int R, int E>
__device__ __forceinline__ constexpr double2 root_c() {
    constexpr int e = E % R;
    if constexpr (R == 6) {
        constexpr double re[6] = {1.0, 0.5, -0.5, -1.0, -0.5, 0.5};
        constexpr double im[6] = {0.0, -kS3, -kS3, 0.0, kS3, kS3};
        return make_double2(re[e], im[e]);
    } else if constexpr (R == 8) {
        constexpr double re[8] = {1.0, kS2, 0.0, -kS2, -1.0, -kS2, 0.0, kS2};
        constexpr double im[8] = {0.0, -kS2, -1.0, -kS2, 0.0, kS2, 1.0, kS2};
        return make_double2(re[e], im[e]);
    } else {  // 10: cos 36 = -c52, sin 36 = s52, cos 72 = c51, sin 72 = s51
        constexpr double re[10] = {1.0, -kC52, kC51, -kC51, kC52, -1.0, kC52, -kC51, kC51, -kC52};
        constexpr double im[10] = {0.0, -kS52, -kS51, -kS51, -kS52, 0.0, kS52, kS51, kS51, kS52};
        return make_double2(re[e], im[e]);
    }
}

// x * w_R^E, the trivial roots (1, -1, -i, i) without arithmetic.
template <int R, int E>
__device__ __forceinline__ double2 mul_root(double2 x) {
    constexpr int e = E % R;
    if constexpr (e == 0) {
        return x;
    } else if constexpr (2 * e == R) {
        return make_double2(-x.x, -x.y);
    } else if constexpr (4 * e == R) {  // -i
        return make_double2(x.y, -x.x);
    } else if constexpr (4 * e == 3 * R) {  // i
        return make_double2(-x.y, x.x);
    } else {
        return cmul(x, root_c<R, E>());
    }
}

// Length R1 R2 DFT of v in place (Cooley-Tukey): Y[r2][k1] = DFT_R1 over r1
// of v[R2 r1 + r2], times w_R^(r2 k1); then X[k1 + R1 k2] = DFT_R2 over r2
// of Y[r2][k1].  All indices compile-time: the values stay in registers.
template <int R1, int R2>
__device__ __forceinline__ void dft_comp(double2 (&v)[R1 * R2]) {
    constexpr int R = R1 * R2;
    double2 y[R];
#pragma unroll
    for (int r2 = 0; r2 < R2; ++r2) {
        double2 t[R1];
#pragma unroll
        for (int r1 = 0; r1 < R1; ++r1) t[r1] = v[R2 * r1 + r2];
        small_dft<R1>(t);
        y[r2 * R1] = t[0];
#pragma unroll
        for (int k1 = 1; k1 < R1; ++k1) {
            double2 z = t[k1];
            // exponent r2 k1 (compile-time after unrolling)
            switch (r2 * k1) {
#define LES_ROOT_CASE(E) \
    case E: z = mul_root<R, E>(z); break;
                LES_ROOT_CASE(0) LES_ROOT_CASE(1) LES_ROOT_CASE(2) LES_ROOT_CASE(3) LES_ROOT_CASE(4)
                LES_ROOT_CASE(5) LES_ROOT_CASE(6) LES_ROOT_CASE(7) LES_ROOT_CASE(8) LES_ROOT_CASE(9)
#undef LES_ROOT_CASE
                default: break;
            }
            y[r2 * R1 + k1] = z;
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        double2 t[R2];
#pragma unroll
        for (int r2 = 0; r2 < R2; ++r2) t[r2] = y[r2 * R1 + k1];
        small_dft<R2>(t);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
}

// One Stockham stage of radix R over npts points (whole lines), a -> b.
// The twiddles of butterfly k of the stage are tws[(r - 1) Ns + k],
// r = 1..R-1: consecutive k, consecutive addresses.
template <int R>
__device__ __forceinline__ void fft_stage(const FftPlan &P, const double2 *a, double2 *b, int npts, int Ns,
                                          const double2 *tws) {
    const int n = P.n, nr = n / R, nb = npts / R;
    const float rnr = 1.0f / (float)nr, rns = 1.0f / (float)Ns;
    for (int t = threadIdx.x; t < nb; t += kFftThreads) {
        const int line = fdiv_small(t, nr, rnr), j = t - line * nr, k = j - fdiv_small(j, Ns, rns) * Ns;
        const double2 *src = a + line * n + j;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 x = src[r * nr];
            v[r] = (r == 0) ? x : cmul(x, __ldg(&tws[(r - 1) * Ns + k]));
        }
        double2 *dst = b + line * n + (j - k) * R + k;
        if constexpr (R <= 5) {
            small_dft<R>(v);
#pragma unroll
            for (int r = 0; r < R; ++r) dst[r * Ns] = v[r];
        } else if constexpr (R == 6 || R == 8 || R == 10) {
            dft_comp<(R == 8 ? 4 : 2), (R == 8 ? 2 : R / 2)>(v);
#pragma unroll
            for (int r = 0; r < R; ++r) dst[r * Ns] = v[r];
        } else {  // V_q = sum_r v_r root^(r q), root = w^(n/R), each stored as it is summed
            const double2 *roots = P.tw + P.troot;
#pragma unroll
            for (int q = 0; q < R; ++q) {
                double2 acc = v[0];
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const double2 root = __ldg(&roots[((r * q) % R) * nr]);
                    acc.x = fma(v[r].x, root.x, fma(-v[r].y, root.y, acc.x));
                    acc.y = fma(v[r].x, root.y, fma(v[r].y, root.x, acc.y));
                }
                dst[q * Ns] = acc;
            }
        }
    }
}

// The rare radices as calls, so that their register demand does not raise
// the common stages'.
template <int R>
__device__ __noinline__ void fft_stage_call(const FftPlan &P, const double2 *a, double2 *b, int npts, int Ns,
                                            const double2 *tws) {
    fft_stage<R>(P, a, b, npts, Ns, tws);
}

// The stages over a (npts points: whole lines), a -> b -> a ...; the
// caller has met a barrier after filling a.  Returns the buffer holding the
// result, after a barrier.
__device__ __forceinline__ double2 *fft_stages(const FftPlan &P, double2 *a, double2 *b, int npts) {
    int Ns = 1;
    for (int s = 0; s < P.nstage; ++s) {
        const int R = P.radix[s];
        const double2 *tws = P.tw + P.tofs[s];
        switch (R) {
            case 2: fft_stage<2>(P, a, b, npts, Ns, tws); break;
            case 3: fft_stage<3>(P, a, b, npts, Ns, tws); break;
            case 4: fft_stage<4>(P, a, b, npts, Ns, tws); break;
            case 5: fft_stage<5>(P, a, b, npts, Ns, tws); break;
            case 6: fft_stage<6>(P, a, b, npts, Ns, tws); break;
            case 8: fft_stage<8>(P, a, b, npts, Ns, tws); break;
            case 10: fft_stage<10>(P, a, b, npts, Ns, tws); break;
            case 7: fft_stage_call<7>(P, a, b, npts, Ns, tws); break;
            case 11: fft_stage_call<11>(P, a, b, npts, Ns, tws); break;
            default: fft_stage_call<13>(P, a, b, npts, Ns, tws); break;
        }
        __syncthreads();
        double2 *tmp = a;
        a = b;
        b = tmp;
        Ns *= R;
    }
    return a;
}

// Forward real-to-complex: nlines (even) lines of n reals (stride n) ->
// n/2 + 1 coefficients each (stride n/2 + 1).  A block loops over groups of
// P.lpb line pairs (a grid of a few blocks per SM); a warp moves one line
// at a time.  stop (may be NULL): skip when *stop is set.
__global__ void __launch_bounds__(kFftThreads, 3) k_fft_r2c(const __grid_constant__ FftPlan P,
                                                            const double *__restrict__ in, double2 *__restrict__ out,
                                                            int nlines, const int *stop) {
    extern __shared__ double2 fsm[];
    if (stop && *stop) return;
    const int n = P.n, nh = n / 2 + 1, npair = nlines / 2, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarp = kFftThreads / 32;
    double2 *za = fsm, *zb = fsm + P.lpb * n;
    double *zr = reinterpret_cast<double *>(za);
    const float rn = 1.0f / (float)n;
    for (int p0 = blockIdx.x * P.lpb; p0 < npair; p0 += gridDim.x * P.lpb) {
        const int pairs = min(P.lpb, npair - p0), tot = 2 * pairs * n;
        const double *src = in + (size_t)2 * p0 * n;
        // the group's lines, kLoadBatch loads of each thread in flight at a time
        for (int t0 = threadIdx.x; t0 < tot; t0 += kLoadBatch * kFftThreads) {
            double x[kLoadBatch];
#pragma unroll
            for (int q = 0; q < kLoadBatch; ++q) {
                const int t = t0 + q * kFftThreads;
                x[q] = t < tot ? src[t] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < kLoadBatch; ++q) {
                const int t = t0 + q * kFftThreads;
                if (t < tot) {
                    const int line = fdiv_small(t, n, rn), i = t - line * n;
                    zr[2 * ((line >> 1) * n + i) + (line & 1)] = x[q];
                }
            }
        }
        __syncthreads();
        const double2 *res = fft_stages(P, za, zb, pairs * n);
        for (int l = warp; l < 2 * pairs; l += nwarp) {
            const double2 *Z = res + (l >> 1) * n;
            double2 *o = out + (size_t)(2 * p0 + l) * nh;
            for (int m = lane; m < nh; m += 32) {
                const double2 a = Z[m], b = Z[m == 0 ? 0 : n - m];
                o[m] = (l & 1) ? make_double2(0.5 * (a.y + b.y), 0.5 * (b.x - a.x))  // (Z_m - conj Z_{n-m}) / 2i
                               : make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y)); // (Z_m + conj Z_{n-m}) / 2
            }
        }
        __syncthreads();
    }
}

// Inverse complex-to-real (unnormalised): x_t = sum_m X_m exp(+2 pi i m t / n)
// for the Hermitian spectrum whose half X_0..X_{n/2} is given (the
// imaginary parts of X_0 and X_{n/2} taken as zero); nlines even.  Lines
// 2p and 2p + 1 go through one FFT: z = conj FFT(conj Z), Z = A + i B.
__global__ void __launch_bounds__(kFftThreads, 3) k_fft_c2r(const __grid_constant__ FftPlan P,
                                                            const double2 *__restrict__ in, double *__restrict__ out,
                                                            int nlines, const int *stop) {
    extern __shared__ double2 fsm[];
    if (stop && *stop) return;
    const int n = P.n, nh = n / 2 + 1, npair = nlines / 2, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nwarp = kFftThreads / 32;
    double2 *za = fsm, *zb = fsm + P.lpb * n;
    const float rnh = 1.0f / (float)nh;
    for (int p0 = blockIdx.x * P.lpb; p0 < npair; p0 += gridDim.x * P.lpb) {
        const int pairs = min(P.lpb, npair - p0), tot = pairs * nh;
        // conj Z_m, Z_m = A_m + i B_m; for m > n/2, A_m = conj A_{n-m}, B_m = conj B_{n-m};
        // kLoadBatch / 2 (A, B) pairs of loads of each thread in flight at a time
        for (int t0 = threadIdx.x; t0 < tot; t0 += (kLoadBatch / 2) * kFftThreads) {
            double2 xa[kLoadBatch / 2], xb[kLoadBatch / 2];
#pragma unroll
            for (int q = 0; q < kLoadBatch / 2; ++q) {
                const int t = t0 + q * kFftThreads;
                if (t < tot) {
                    const int p = fdiv_small(t, nh, rnh), m = t - p * nh;
                    const double2 *A = in + (size_t)2 * (p0 + p) * nh;
                    xa[q] = A[m];
                    xb[q] = A[nh + m];
                }
            }
#pragma unroll
            for (int q = 0; q < kLoadBatch / 2; ++q) {
                const int t = t0 + q * kFftThreads;
                if (t < tot) {
                    const int p = fdiv_small(t, nh, rnh), m = t - p * nh;
                    const double2 x = xa[q], y = xb[q];
                    double2 *z = za + p * n;
                    if (m == 0 || 2 * m == n) {
                        z[m] = make_double2(x.x, -y.x);
                    } else {
                        z[m] = make_double2(x.x - y.y, -(x.y + y.x));
                        z[n - m] = make_double2(x.x + y.y, x.y - y.x);
                    }
                }
            }
        }
        __syncthreads();
        const double2 *res = fft_stages(P, za, zb, pairs * n);
        for (int l = warp; l < 2 * pairs; l += nwarp) {
            const double2 *w = res + (l >> 1) * n;
            double *dst = out + (size_t)(2 * p0 + l) * n;
            if (l & 1) {
                for (int i = lane; i < n; i += 32) dst[i] = -w[i].y;
            } else {
                for (int i = lane; i < n; i += 32) dst[i] = w[i].x;
            }
        }
        __syncthreads();
    }
}

// Host side.  The plan of lines of length n (even, at most kFftPoints):
// radices largest first (4, 5, 3, 2, 7, 11, 13), the twiddle table's layout,
// line pairs per block so a block holds about kFftPoints points, and a grid
// of 3 blocks per SM (nsm SMs) that loop over the line groups.  Returns the
// table's length in double2 entries (P.tw still to be set), or -1.
inline int fft_plan(int n, int nsm, FftPlan &P) {
    P = FftPlan{};
    if (n < 2 || n % 2 || n > kFftPoints) return -1;
    P.n = n;
    int m = n, ofs = 0, Ns = 1;
    for (int r : {10, 8, 6, 4, 5, 3, 2, 7, 11, 13})
        while (m % r == 0 && m > 1) {
            if (P.nstage == kFftMaxStages) return -1;
            P.tofs[P.nstage] = ofs;
            P.radix[P.nstage++] = r;
            ofs += (r - 1) * Ns;
            Ns *= r;
            m /= r;
        }
    if (m != 1) return -1;
    P.troot = ofs;
    P.lpb = std::max(1, kFftPoints / n);
    P.blocks = 3 * std::max(nsm, 1);
    return ofs + n;
}

// The table fft_plan laid out: stage s (Ns points combined, radix R) entry
// (r - 1) Ns + k = w^(r k n / (Ns R)), then w^k, k < n; w = exp(-2 pi i / n).
inline std::vector<double2> fft_twiddles(const FftPlan &P) {
    const double two_pi = 6.28318530717958647693;
    const int n = P.n;
    auto w = [&](long long e) {
        const double a = two_pi * (double)(e % n) / n;
        return make_double2(std::cos(a), -std::sin(a));
    };
    std::vector<double2> t(P.troot + n);
    int Ns = 1;
    for (int s = 0; s < P.nstage; ++s) {
        const int R = P.radix[s], stride = n / (Ns * R);
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < Ns; ++k) t[P.tofs[s] + (r - 1) * Ns + k] = w((long long)r * k * stride);
        Ns *= R;
    }
    for (int k = 0; k < n; ++k) t[P.troot + k] = w(k);
    return t;
}

}  // namespace
}  // namespace les
