// les_adjoint.cuh -- reverse-mode (adjoint) kernels of the routines whose
// map is linear: press.f95:49-146 run with a fixed number of SOR iterations
// (the count a forward call executed), velnw, feedbf (masks fixed), adam.
//
// With that count fixed the routine is a linear map of its inputs: bondfg
// (bondFG.f95:15-31) copies and clears ghost faces of f, g, h; rhs is the
// divergence of (f, g, h) plus that of (u, v, w) over dt (press.f95:49-69);
// rhsav, the dx1*dy1*dzn-weighted mean of rhs, is subtracted (press.f95:
// 70-82); each SOR half-sweep replaces the cells of one colour by
//     p_c <- (1 - omega) p_c + omega cn1_c (sum_nb c_nb p_nb - rhs_c)
// reading only other-colour cells and ghosts (press.f95:89-98), followed by
// boundp1 (ghost copies in i, then j), and each iteration by boundp2 (k);
// finally pav, the weighted mean of p, is subtracted and the ghosts copied
// again (press.f95:123-146).  The adjoint applies the transposes in reverse
// order.  A transposed half-sweep scales the swept cells' adjoints by
// (1 - omega), moves -omega cn1_c times them into the rhs adjoint, and adds
// omega cn1_c c_nb times them to every neighbour the forward sweep read: the
// other colour's cells and the ghost faces.  It reads one adjoint buffer
// and writes the other, so every location is a gather.
//
// Arrays use the box layout of the forward kernels (IX), with p's Fortran
// range 0..im+2, 0..jm+2, 0..km+1; locations the routine never touches keep
// their adjoint.  Sums (the two mean removals) are FP64 in a fixed order.
#pragma once

#include "les_dev.cuh"

namespace les {
namespace {

constexpr int kAdjBX = 32, kAdjBY = 8;

// boundp2 transposed (boundp.f95:5-21): p(.,.,0) = p(.,.,1), then
// p(.,.,km+1) = p(.,.,km), for i = 0..im+1, j = 0..jm+1.
__global__ void k_adj_boundp2(Geo g, float *pb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x, ni = g.im + 2;
    if (t >= ni * (g.jm + 2)) return;
    const int i = t % ni, j = t / ni;
    float &a0 = pb[IX(g, i, j, 0)], &a1 = pb[IX(g, i, j, 1)];
    float &am = pb[IX(g, i, j, g.km)], &am1 = pb[IX(g, i, j, g.km + 1)];
    am += am1;
    am1 = 0.0f;
    a1 += a0;
    a0 = 0.0f;
}

// boundp1 transposed, second loop (boundp.f95:36-42): p(i,0,k) = p(i,jm,k),
// then p(i,jm+1,k) = p(i,1,k), for i = 0..im+1, k = 0..km+1.
__global__ void k_adj_boundp1_j(Geo g, float *pb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x, ni = g.im + 2;
    if (t >= ni * (g.km + 2)) return;
    const int i = t % ni, k = t / ni;
    float &a0 = pb[IX(g, i, 0, k)], &a1 = pb[IX(g, i, 1, k)];
    float &am = pb[IX(g, i, g.jm, k)], &am1 = pb[IX(g, i, g.jm + 1, k)];
    a1 += am1;
    am1 = 0.0f;
    am += a0;
    a0 = 0.0f;
}

// boundp1 transposed, first loop (boundp.f95:28-34): p(0,j,k) = p(1,j,k),
// then p(im+1,j,k) = p(im,j,k), for j = 0..jm+1, k = 0..km+1.
__global__ void k_adj_boundp1_i(Geo g, float *pb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x, nj = g.jm + 2;
    if (t >= nj * (g.km + 2)) return;
    const int j = t % nj, k = t / nj;
    float &a0 = pb[IX(g, 0, j, k)], &a1 = pb[IX(g, 1, j, k)];
    float &am = pb[IX(g, g.im, j, k)], &am1 = pb[IX(g, g.im + 1, j, k)];
    am += am1;
    am1 = 0.0f;
    a1 += a0;
    a0 = 0.0f;
}

// One SOR half-sweep of colour nrd transposed: in -> out over p's range;
// rhsb of the swept cells accumulates.  Cell (i,j,k) is swept when
// i + j + k + nrd is odd (press.f95:91, i = 1 + mod(k+j+nrd, 2), step 2).
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_sweep(Geo g, const float *in, float *out, float *rhsb,
                                                              const float *cn1, int nrd, float omega) {
    const int i = blockIdx.x * kAdjBX + threadIdx.x, j = blockIdx.y * kAdjBY + threadIdx.y, k = blockIdx.z;
    if (i > g.im + 2 || j > g.jm + 2) return;
    const int im = g.im, jm = g.jm, km = g.km;
    const int c = IX(g, i, j, k);
    const float v = in[c];
    const bool ii = i >= 1 && i <= im, jj = j >= 1 && j <= jm, kk = k >= 1 && k <= km;
    // what the forward sweep at swept cell (a,b,d) took from this location
    // through coefficient coef
    auto from = [&](int a, int b, int d, float coef) {
        const int q = IX(g, a, b, d);
        return omega * (cn1[q] * coef) * in[q];
    };
    auto swept = [&](int a, int b, int d) { return ((a + b + d + nrd) & 1) != 0; };
    float r = v;
    if (ii && jj && kk) {
        if (swept(i, j, k)) {
            rhsb[c] -= (omega * cn1[c]) * v;
            r = (1.0f - omega) * v;
        } else {  // every interior neighbour was swept
            if (i > 1) r += from(i - 1, j, k, g.cn2l[i - 1]);
            if (i < im) r += from(i + 1, j, k, g.cn2s[i + 1]);
            if (j > 1) r += from(i, j - 1, k, g.cn3l[j - 1]);
            if (j < jm) r += from(i, j + 1, k, g.cn3s[j + 1]);
            if (k > 1) r += from(i, j, k - 1, g.cn4l[k - 1]);
            if (k < km) r += from(i, j, k + 1, g.cn4s[k + 1]);
        }
    } else if (jj && kk && i == 0) {
        if (swept(1, j, k)) r += from(1, j, k, g.cn2s[1]);
    } else if (jj && kk && i == im + 1) {
        if (swept(im, j, k)) r += from(im, j, k, g.cn2l[im]);
    } else if (ii && kk && j == 0) {
        if (swept(i, 1, k)) r += from(i, 1, k, g.cn3s[1]);
    } else if (ii && kk && j == jm + 1) {
        if (swept(i, jm, k)) r += from(i, jm, k, g.cn3l[jm]);
    } else if (ii && jj && k == 0) {
        if (swept(i, j, 1)) r += from(i, j, 1, g.cn4s[1]);
    } else if (ii && jj && k == km + 1) {
        if (swept(i, j, km)) r += from(i, j, km, g.cn4l[km]);
    }
    out[c] = r;
}

// Interior sum of x in FP64: one partial per 32 x 8 tile of a plane (fixed
// tree), then k_adj_sum_final adds the partials in a fixed order.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_sum_part(Geo g, const float *x, double *part) {
    __shared__ double s[kAdjBX * kAdjBY];
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z, t = threadIdx.y * kAdjBX + threadIdx.x;
    s[t] = (i <= g.im && j <= g.jm) ? (double)x[IX(g, i, j, k)] : 0.0;
    __syncthreads();
    for (int h = kAdjBX * kAdjBY / 2; h > 0; h >>= 1) {
        if (t < h) s[t] += s[t + h];
        __syncthreads();
    }
    if (t == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s[0];
}
__global__ void __launch_bounds__(1024) k_adj_sum_final(const double *part, int n, double *out) {
    __shared__ double s[1024];
    double a = 0.0;
    for (int b = threadIdx.x; b < n; b += 1024) a += part[b];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int h = 512; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// A weighted-mean removal x -= (sum w x)/W (w = dx1*dy1*dzn) transposed:
// x_c -= w_c * (sum x) / W over the interior, *sum from k_adj_sum_final.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_mean_sub(Geo g, float *x, const double *sum, double area) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const double wc = (double)(g.dx1[i] * g.dy1[j] * g.dzn[k]);
    float &a = x[IX(g, i, j, k)];
    a = (float)((double)a - wc * (*sum / area));
}

// rhs of press.f95:54-68 transposed: each location (i,j,k), 0 <= i <= im,
// 0 <= j <= jm, 0 <= k <= km, gathers the rhs adjoints of the (at most two)
// cells whose divergence read it; (u, v, w) take them over dt.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_rhs(Geo g, const float *rhsb, float *ub, float *vb,
                                                            float *wb, float *fb, float *gb, float *hb, float dt) {
    const int i = blockIdx.x * kAdjBX + threadIdx.x, j = blockIdx.y * kAdjBY + threadIdx.y, k = blockIdx.z;
    const int im = g.im, jm = g.jm, km = g.km;
    if (i > im || j > jm) return;
    const int c = IX(g, i, j, k);
    auto rb = [&](int a, int b, int d) { return rhsb[IX(g, a, b, d)]; };
    if (j >= 1 && k >= 1) {  // u(i), f(i): rhs(i) with +1/dx1(i), rhs(i+1) with -1/dx1(i+1)
        float x = 0.0f;
        if (i >= 1) x += rb(i, j, k) / g.dx1[i];
        if (i < im) x -= rb(i + 1, j, k) / g.dx1[i + 1];
        fb[c] += x;
        ub[c] += x / dt;
    }
    if (i >= 1 && k >= 1) {
        float y = 0.0f;
        if (j >= 1) y += rb(i, j, k) / g.dy1[j];
        if (j < jm) y -= rb(i, j + 1, k) / g.dy1[j + 1];
        gb[c] += y;
        vb[c] += y / dt;
    }
    if (i >= 1 && j >= 1) {
        float z = 0.0f;
        if (k >= 1) z += rb(i, j, k) / g.dzn[k];
        if (k < km) z -= rb(i, j, k + 1) / g.dzn[k + 1];
        hb[c] += z;
        wb[c] += z / dt;
    }
}

// The forward overwrites rhs on the interior: its input adjoint there is 0.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_zero_interior(Geo g, float *x) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    if (i > g.im || j > g.jm) return;
    x[IX(g, i, j, 1 + blockIdx.z)] = 0.0f;
}

// bondfg transposed (bondFG.f95:15-31): f(0,j,k) = f(1,j,k); g(i,0,k) =
// g(i,jm,k); h(i,j,0) = h(i,j,km) = 0.
__global__ void k_adj_bondfg(Geo g, float *fb, float *gb, float *hb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nf = (long long)g.jm * g.km, ng = (long long)g.im * g.km, nh = (long long)g.im * g.jm;
    if (t < nf) {
        const int j = 1 + (int)(t % g.jm), k = 1 + (int)(t / g.jm);
        fb[IX(g, 1, j, k)] += fb[IX(g, 0, j, k)];
        fb[IX(g, 0, j, k)] = 0.0f;
    } else if (t < nf + ng) {
        const long long r = t - nf;
        const int i = 1 + (int)(r % g.im), k = 1 + (int)(r / g.im);
        gb[IX(g, i, g.jm, k)] += gb[IX(g, i, 0, k)];
        gb[IX(g, i, 0, k)] = 0.0f;
    } else if (t < nf + ng + nh) {
        const long long r = t - nf - ng;
        const int i = 1 + (int)(r % g.im), j = 1 + (int)(r / g.im);
        hb[IX(g, i, j, g.km)] = 0.0f;
        hb[IX(g, i, j, 0)] = 0.0f;
    }
}

// velnw.f95:27-59 transposed.  The forward adds dt*(f - (p(+1) - p)/ro/ds)
// to u, v (all k) and w (k <= km-1); u, v, w keep their adjoints, f, g, h
// gain dt times them, and each p location gathers from the (at most two)
// faces per axis whose pressure difference read it.  Locations: p's
// 1..im+1, 1..jm+1, 1..km.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_velnw(Geo g, const float *ub, const float *vb,
                                                              const float *wb, float *pb, float *fb, float *gb,
                                                              float *hb, float dt) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    const int im = g.im, jm = g.jm, km = g.km;
    if (i > im + 1 || j > jm + 1) return;
    const bool ii = i <= im, jj = j <= jm;
    const float ro = g.ro;
    auto at = [&](const float *a, int x, int y, int z) { return a[IX(g, x, y, z)]; };
    float r = 0.0f;
    if (jj) {
        if (i > 1) r -= ((dt * at(ub, i - 1, j, k)) / ro) / g.dxs[i - 1];
        if (ii) r += ((dt * at(ub, i, j, k)) / ro) / g.dxs[i];
    }
    if (ii) {
        if (j > 1) r -= ((dt * at(vb, i, j - 1, k)) / ro) / g.dys[j - 1];
        if (jj) r += ((dt * at(vb, i, j, k)) / ro) / g.dys[j];
    }
    if (ii && jj) {
        if (k > 1) r -= ((dt * at(wb, i, j, k - 1)) / ro) / g.dzs[k - 1];
        if (k < km) r += ((dt * at(wb, i, j, k)) / ro) / g.dzs[k];
    }
    const int c = IX(g, i, j, k);
    pb[c] += r;
    if (ii && jj) {
        fb[c] += dt * ub[c];
        gb[c] += dt * vb[c];
        if (k < km) hb[c] += dt * wb[c];
    }
}

// feedbf.f95:38-67 transposed, per interior cell and component:
//   usum' = (usum + u) m;  fx = (alpha usum') dt + (beta u) m;  f' = f + fx.
// f keeps its adjoint; fx's is spent (fx is overwritten); usum and u gather.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_feedbf(Geo g, Fields F, float *fxb, float *fyb, float *fzb,
                                                               float alpha, float dt, float beta) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    auto comp = [&](float *sumb, float *vb, const float *mask, float *xb, const float *fb) {
        const float m = mask[c];
        const float t = xb[c] + fb[c];
        const float sb = sumb[c] + (alpha * dt) * t;
        vb[c] += (beta * m) * t + m * sb;
        sumb[c] = m * sb;
        xb[c] = 0.0f;
    };
    comp(F.usum, F.u, F.bmask, fxb, F.f);
    comp(F.vsum, F.v, F.cmask, fyb, F.g);
    comp(F.wsum, F.w, F.dmask, fzb, F.h);
}

// adam.f95:32-46 transposed: f' = 1.5 f - 0.5 fold, fold' = f.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_adam(Geo g, Fields F) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    float *cur[3] = {F.f, F.g, F.h}, *old[3] = {F.fold, F.gold, F.hold};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float b = cur[a][c], ob = old[a][c];
        cur[a][c] = 1.5f * b + ob;
        old[a][c] = -0.5f * b;
    }
}

}  // namespace
}  // namespace les
