// les_fft.cuh -- batched FP64 FFTs of contiguous lines for the spectral solve
// of the refined press (les_spectral.cuh): real-to-complex forward (the
// first n/2 + 1 coefficients) and complex-to-real inverse (unnormalised,
// the input taken as the half spectrum of a real line).
//
// Mixed-radix Stockham autosort FFT in shared memory (radices 4, 5, 3, 2,
// 7 and any other prime factor of n, largest stages first): a stage of
// radix R with Ns points already combined reads v_r = a[j + r n/R] times the
// twiddle w^(r (j mod Ns) n/(Ns R)), w = exp(-2 pi i / n), takes their
// length-R DFT (roots from the same table, w^(n/R)), and writes it to
// b[(j div Ns) Ns R + (j mod Ns) + r Ns]; after the last stage the line is
// in natural order.  A block transforms several lines at once; the twiddles
// exp(-2 pi i k / n), k < n, come from a host-built table.
#pragma once

#include "les_dev.cuh"

namespace les {
namespace {

constexpr int kFftMaxStages = 24, kFftMaxRadix = 16, kFftThreads = 256, kFftPoints = 2048;

struct FftPlan {
    int n, nstage;
    int radix[kFftMaxStages];
    const double2 *tw;  // exp(-2 pi i k / n), k = 0..n-1
    int lpb;            // lines per block
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Length-R DFT of v (in place): w_q = sum_r v_r root^(r q), root = w^(n/R).
template <int R>
__device__ __forceinline__ void small_dft(double2 (&v)[R], const double2 *tw, int rootstep) {
    if constexpr (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = make_double2(a.x + b.x, a.y + b.y);
        v[1] = make_double2(a.x - b.x, a.y - b.y);
    } else if constexpr (R == 4) {  // roots 1, -i, -1, i
        const double2 s02 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
        const double2 d02 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
        const double2 s13 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
        const double2 d13 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
        v[0] = make_double2(s02.x + s13.x, s02.y + s13.y);
        v[2] = make_double2(s02.x - s13.x, s02.y - s13.y);
        v[1] = make_double2(d02.x + d13.y, d02.y - d13.x);  // d02 - i d13
        v[3] = make_double2(d02.x - d13.y, d02.y + d13.x);  // d02 + i d13
    } else {
        double2 w[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            double2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const double2 root = tw[((r * q) % R) * rootstep];
                acc.x += v[r].x * root.x - v[r].y * root.y;
                acc.y += v[r].x * root.y + v[r].y * root.x;
            }
            w[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = w[q];
    }
}

// One Stockham stage of radix R over a block's lines: a -> b.
template <int R>
__device__ __forceinline__ void fft_stage(const FftPlan &P, const double2 *a, double2 *b, int lines, int Ns) {
    const int n = P.n, nr = n / R, stride = n / (Ns * R);
    for (int t = threadIdx.x; t < lines * nr; t += blockDim.x) {
        const int line = t / nr, j = t - line * nr, k = j % Ns;
        const double2 *src = a + line * n;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 x = src[j + r * nr];
            v[r] = (r == 0 || k == 0) ? x : cmul(x, P.tw[r * k * stride]);  // r k stride < n
        }
        small_dft<R>(v, P.tw, nr);
        double2 *dst = b + line * n + (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[r * Ns] = v[r];
    }
}

// A stage of any other (prime) radix, R <= kFftMaxRadix.
__device__ void fft_stage_any(const FftPlan &P, const double2 *a, double2 *b, int lines, int Ns, int R) {
    const int n = P.n, nr = n / R, stride = n / (Ns * R);
    for (int t = threadIdx.x; t < lines * nr; t += blockDim.x) {
        const int line = t / nr, j = t - line * nr, k = j % Ns;
        const double2 *src = a + line * n;
        double2 *dst = b + line * n + (j / Ns) * Ns * R + k;
        for (int q = 0; q < R; ++q) {
            double2 acc = make_double2(0.0, 0.0);
            for (int r = 0; r < R; ++r) {
                const double2 x = src[j + r * nr];
                const double2 v = (r == 0 || k == 0) ? x : cmul(x, P.tw[r * k * stride]);
                const double2 root = P.tw[((r * q) % R) * nr];
                acc.x += v.x * root.x - v.y * root.y;
                acc.y += v.x * root.y + v.y * root.x;
            }
            dst[q * Ns] = acc;
        }
    }
}

// The stages of one block's lines, a -> b -> a ...; returns the buffer
// holding the result.
__device__ double2 *fft_stages(const FftPlan &P, double2 *a, double2 *b, int lines) {
    int Ns = 1;
    for (int s = 0; s < P.nstage; ++s) {
        const int R = P.radix[s];
        __syncthreads();
        switch (R) {
            case 2: fft_stage<2>(P, a, b, lines, Ns); break;
            case 3: fft_stage<3>(P, a, b, lines, Ns); break;
            case 4: fft_stage<4>(P, a, b, lines, Ns); break;
            case 5: fft_stage<5>(P, a, b, lines, Ns); break;
            case 7: fft_stage<7>(P, a, b, lines, Ns); break;
            default: fft_stage_any(P, a, b, lines, Ns, R); break;
        }
        double2 *tmp = a;
        a = b;
        b = tmp;
        Ns *= R;
    }
    __syncthreads();
    return a;
}

// Forward real-to-complex: lines of n reals (stride n) -> n/2 + 1
// coefficients (stride n/2 + 1).  stop (may be NULL): skip when *stop is set.
__global__ void __launch_bounds__(kFftThreads) k_fft_r2c(const __grid_constant__ FftPlan P, const double *in, double2 *out, int nlines,
                                                         const int *stop) {
    extern __shared__ double2 fsm[];
    if (stop && *stop) return;
    const int n = P.n, nh = n / 2 + 1;
    const int l0 = blockIdx.x * P.lpb, lines = min(P.lpb, nlines - l0);
    if (lines <= 0) return;
    double2 *a = fsm, *b = fsm + P.lpb * n;
    for (int t = threadIdx.x; t < lines * n; t += blockDim.x) a[t] = make_double2(in[(size_t)l0 * n + t], 0.0);
    const double2 *res = fft_stages(P, a, b, lines);
    for (int t = threadIdx.x; t < lines * nh; t += blockDim.x) {
        const int line = t / nh, m = t - line * nh;
        out[(size_t)(l0 + line) * nh + m] = res[line * n + m];
    }
}

// Inverse complex-to-real (unnormalised): x_t = sum_m X_m exp(+2 pi i m t / n)
// for the Hermitian spectrum whose half X_0..X_{n/2} is given (the
// imaginary parts of X_0 and X_{n/2} taken as zero): x = Re FFT(conj X).
__global__ void __launch_bounds__(kFftThreads) k_fft_c2r(const __grid_constant__ FftPlan P, const double2 *in, double *out, int nlines,
                                                         const int *stop) {
    extern __shared__ double2 fsm[];
    if (stop && *stop) return;
    const int n = P.n, nh = n / 2 + 1;
    const int l0 = blockIdx.x * P.lpb, lines = min(P.lpb, nlines - l0);
    if (lines <= 0) return;
    double2 *a = fsm, *b = fsm + P.lpb * n;
    for (int t = threadIdx.x; t < lines * n; t += blockDim.x) {
        const int line = t / n, m = t - line * n;
        const double2 *X = in + (size_t)(l0 + line) * nh;
        double2 v;
        if (m == 0 || 2 * m == n)
            v = make_double2(X[m].x, 0.0);
        else if (m < nh)
            v = make_double2(X[m].x, -X[m].y);
        else
            v = X[n - m];
        a[t] = v;
    }
    const double2 *res = fft_stages(P, a, b, lines);
    for (int t = threadIdx.x; t < lines * n; t += blockDim.x) out[(size_t)l0 * n + t] = res[t].x;
}

}  // namespace
}  // namespace les
