// les_spectral.cuh -- FP64 spectral solve of the refined press's operator
// A (les_refine.cuh) on grids with uniform x and y spacing.
//
// There A = Ax + Ay + Az exactly: Ax = c2 (p_e + p_w - 2p) with the Neumann
// ghosts has the DCT-II vectors cos(pi m (i - 1/2) / im) as eigenvectors
// (eigenvalue 2 c2 (cos(pi m / im) - 1)); Ay, periodic, the Fourier modes
// (2 c3 (cos(2 pi n / jm) - 1)); Az is tridiagonal in k.  So A e = r is:
// a DCT-II along i, a real DFT along j, one tridiagonal solve in k per mode
// (m, n) with the diagonal shifted by the two eigenvalues, and the inverse
// transforms.  The DCT-II of an even-length line is one real FFT of the
// line's values taken in even-then-reversed-odd order, twiddled by
// exp(-i pi m / 2N) (J. Makhoul, IEEE Trans. ASSP 28(1), 1980), and its
// inverse the reverse.  The FFTs are les_fft.cuh's (FP64, mixed radix); the
// twiddles, transposes, tridiagonal solves and the correction are these
// kernels.  The whole tail is captured in the step graph: corrections after
// the tolerance is met return at once on the device (Ref64::stop).
//
// Layouts (dense, FP64): r and v lines [k][j][pos] (makhoul_pos order);
// V = FFT of a line [k][j][0..im/2]; X [k][m][j] (j contiguous, for the
// DFT along j); Y [k][m][0..jm/2].  The mode (0,0) has the singular
// Neumann tridiagonal: its last equation is dropped and e(km) set to 0
// (the right-hand side is compatible, les_refine.cuh).
#pragma once

#include "les_refine.cuh"

namespace les {
namespace {

constexpr int kSpecT = 32;

// The transposes and the correction loop over k planes blockIdx.z,
// blockIdx.z + gridDim.z, ... so that a skipped correction (*stop set)
// launches few blocks.

// X[k][m][j] = Re(exp(-i pi m / 2N) V_m) with V_m = conj(V_{N-m}) for m > N/2.
__global__ void __launch_bounds__(kSpecT * 8) k_spec_fwd(const double2 *V, double *X, const double2 *tw, int im,
                                                           int jm, int km, const int *stop) {
    __shared__ double t[kSpecT][kSpecT + 1];
    if (*stop) return;
    const int m0 = blockIdx.x * kSpecT, j0 = blockIdx.y * kSpecT, nh = im / 2 + 1;
    for (int k = blockIdx.z; k < km; k += gridDim.z) {
        for (int r = threadIdx.y; r < kSpecT; r += blockDim.y) {
            const int j = j0 + r, m = m0 + threadIdx.x;
            double val = 0.0;
            if (j < jm && m < im) {
                const double2 *line = V + ((size_t)k * jm + j) * nh;
                double2 z = (m <= im / 2) ? line[m] : line[im - m];
                if (m > im / 2) z.y = -z.y;
                val = tw[m].x * z.x + tw[m].y * z.y;
            }
            t[r][threadIdx.x] = val;
        }
        __syncthreads();
        for (int r = threadIdx.y; r < kSpecT; r += blockDim.y) {
            const int m = m0 + r, j = j0 + threadIdx.x;
            if (m < im && j < jm) X[((size_t)k * im + m) * jm + j] = t[threadIdx.x][r];
        }
        __syncthreads();
    }
}

// V_m = exp(i pi m / 2N) (X_m - i X_{N-m}), m = 0..N/2, X_N = 0; from
// X[k][m][j] to the lines [k][j][m].
__global__ void __launch_bounds__(kSpecT * 8) k_spec_inv(const double *X, double2 *V, const double2 *tw, int im,
                                                           int jm, int km, const int *stop) {
    __shared__ double ta[kSpecT][kSpecT + 1], tb[kSpecT][kSpecT + 1];
    if (*stop) return;
    const int m0 = blockIdx.x * kSpecT, j0 = blockIdx.y * kSpecT, nh = im / 2 + 1;
    for (int k = blockIdx.z; k < km; k += gridDim.z) {
        for (int r = threadIdx.y; r < kSpecT; r += blockDim.y) {
            const int m = m0 + r, j = j0 + threadIdx.x;
            double a = 0.0, b = 0.0;
            if (m < nh && j < jm) {
                a = X[((size_t)k * im + m) * jm + j];
                b = (m == 0) ? 0.0 : X[((size_t)k * im + (im - m)) * jm + j];
            }
            ta[r][threadIdx.x] = a;
            tb[r][threadIdx.x] = b;
        }
        __syncthreads();
        for (int r = threadIdx.y; r < kSpecT; r += blockDim.y) {
            const int j = j0 + r, m = m0 + threadIdx.x;
            if (m < nh && j < jm) {
                const double a = ta[threadIdx.x][r], b = tb[threadIdx.x][r];
                const double c = tw[m].x, s = tw[m].y;
                V[((size_t)k * jm + j) * nh + m] = make_double2(c * a + s * b, s * a - c * b);
            }
        }
        __syncthreads();
    }
}

// One tridiagonal solve in k per mode (m, n) (Thomas), in place on Y; C
// holds the modified super-diagonal.  zsub/zdiag/zsup: Az with its Neumann
// rows; lx, ly: the x and y eigenvalues.  The loads of kTriAhead levels are
// issued before their sweep steps (the sweeps are a serial chain per mode).
constexpr int kTriAhead = 8;
__global__ void __launch_bounds__(128) k_spec_tridiag(double2 *__restrict__ Y, double *__restrict__ C,
                                                      const double *lx, const double *ly, const double *zsub,
                                                      const double *zdiag, const double *zsup, int im, int jh, int km,
                                                      const Ref64 *R) {
    if (R->stop) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)im * jh) return;
    const int m = (int)(t / jh), n = (int)(t % jh);
    const double lam = lx[m] + ly[n];
    const size_t st = (size_t)im * jh;
    const int kn = (m == 0 && n == 0) ? km - 1 : km;
    double cprev = 0.0;
    double2 dprev = make_double2(0.0, 0.0);
    for (int k0 = 0; k0 < kn; k0 += kTriAhead) {
        double2 d[kTriAhead];
#pragma unroll
        for (int q = 0; q < kTriAhead; ++q)
            if (k0 + q < kn) d[q] = Y[(k0 + q) * st + t];
#pragma unroll
        for (int q = 0; q < kTriAhead; ++q) {
            const int k = k0 + q;
            if (k < kn) {
                const double a = (k > 0) ? zsub[k] : 0.0;
                const double c = (k < kn - 1) ? zsup[k] : 0.0;
                const double inv = 1.0 / (zdiag[k] + lam - a * cprev);
                const double cp = c * inv;
                d[q].x = (d[q].x - a * dprev.x) * inv;
                d[q].y = (d[q].y - a * dprev.y) * inv;
                Y[k * st + t] = d[q];
                C[k * st + t] = cp;
                cprev = cp;
                dprev = d[q];
            }
        }
    }
    if (kn < km) Y[(size_t)(km - 1) * st + t] = make_double2(0.0, 0.0);
    double2 x = dprev;
    for (int k0 = kn - 2; k0 >= 0; k0 -= kTriAhead) {
        double2 d[kTriAhead];
        double cp[kTriAhead];
#pragma unroll
        for (int q = 0; q < kTriAhead; ++q)
            if (k0 - q >= 0) {
                d[q] = Y[(k0 - q) * st + t];
                cp[q] = C[(k0 - q) * st + t];
            }
#pragma unroll
        for (int q = 0; q < kTriAhead; ++q)
            if (k0 - q >= 0) {
                x.x = d[q].x - cp[q] * x.x;
                x.y = d[q].y - cp[q] * x.y;
                Y[(k0 - q) * st + t] = x;
            }
    }
}

// p64 += scale * e on the interior, e from the inverse transforms' lines.
__global__ void __launch_bounds__(kRedNT) k_spec_correct(Geo g, double *__restrict__ p64, const double *__restrict__ v,
                                                          double scale, Ref64 *R) {
    if (R->stop) return;
    const int i = 1 + blockIdx.x * kRedBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kRedBY + threadIdx.y;
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0)
        R->outer += 1;
    if (i > g.im || j > g.jm) return;
    for (int k = 1 + blockIdx.z; k <= g.km; k += gridDim.z) {
        const int c = IX(g, i, j, k);
        p64[c] = p64[c] + scale * v[((size_t)(k - 1) * g.jm + (j - 1)) * g.im + makhoul_pos(i, g.im)];
    }
}

}  // namespace
}  // namespace les
