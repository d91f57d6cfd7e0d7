// les_adjoint.cuh -- reverse-mode (adjoint) kernels: of the routines whose
// map is linear, press.f95:49-146 run with a fixed number of SOR iterations
// (the count a forward call executed), velnw, feedbf (masks fixed), adam;
// and of les (at the forward state, below).
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

// boundp1 transposed (boundp.f95:23-44), one block per plane k = 0..km+1:
// the second loop's copies first (p(i,0,k) = p(i,jm,k), then
// p(i,jm+1,k) = p(i,1,k), i = 0..im+1: in reverse, row jm+1 into row 1, row 0
// into row jm), then, after the block's barrier, the first loop's
// (p(0,j,k) = p(1,j,k), then p(im+1,j,k) = p(im,j,k), j = 0..jm+1: column
// im+1 into column im, column 0 into column 1).
__global__ void __launch_bounds__(256) k_adj_boundp1(Geo g, float *pb) {
    const int k = blockIdx.x;
    for (int i = threadIdx.x; i <= g.im + 1; i += blockDim.x) {
        float &a0 = pb[IX(g, i, 0, k)], &a1 = pb[IX(g, i, 1, k)];
        float &am = pb[IX(g, i, g.jm, k)], &am1 = pb[IX(g, i, g.jm + 1, k)];
        a1 += am1;
        am1 = 0.0f;
        am += a0;
        a0 = 0.0f;
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= g.jm + 1; j += blockDim.x) {
        float &a0 = pb[IX(g, 0, j, k)], &a1 = pb[IX(g, 1, j, k)];
        float &am = pb[IX(g, g.im, j, k)], &am1 = pb[IX(g, g.im + 1, j, k)];
        am += am1;
        am1 = 0.0f;
        a1 += a0;
        a0 = 0.0f;
    }
}

// One SOR half-sweep of colour nrd transposed: in -> out over p's range;
// rhsb of the swept cells accumulates.  Cell (i,j,k) is swept when
// i + j + k + nrd is odd (press.f95:91, i = 1 + mod(k+j+nrd, 2), step 2).
// FOLDK: the transposed boundp2 of the iteration (planes km+1 and 0 into km
// and 1, after which both are zero) is applied to the reads: a linear map
// along k, it commutes with the transposed boundp1, which works within
// planes, so the boundp1 that runs before this half-sweep may come first.
// Only planes k <= 2 and k >= km-1 read plane 1 or km (their own or a
// neighbour's), so only their blocks take the folding body (the plane is
// the block's z, one path per block); neighbours are addressed by offsets
// from the cell's index.
template <bool FOLD>
__device__ __forceinline__ void adj_sweep_cell(const Geo &g, const float *__restrict__ in, float *__restrict__ out,
                                               float *__restrict__ rhsb, const float *__restrict__ cn1, int nrd,
                                               float omega, int i, int j, int k) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int c = IX(g, i, j, k);
    const int sy = g.si, sz = g.si * g.sj;
#ifdef LES_CHECKED
    auto nb = [&](int di, int dj, int dk) { return IX(g, i + di, j + dj, k + dk); };
#else
    auto nb = [&](int di, int dj, int dk) { return c + di + sy * dj + sz * dk; };
#endif
    // in at box index x of plane d, with the fold of planes km+1 and 0
    // (every location read here lies in boundp2's range i <= im+1, j <= jm+1)
    auto ldx = [&](int x, int d) {
        float v = in[x];
        if (FOLD) {
            if (d == km) v += in[x + sz];
            if (d == 1) v += in[x - sz];
        }
        return v;
    };
    // (boundp2 covers i = 0..im+1, j = 0..jm+1; p's last row and column
    // i = im+2, j = jm+2 pass through)
    const bool inb = i <= im + 1 && j <= jm + 1;
    const float v = (FOLD && inb) ? ((k == 0 || k == km + 1) ? 0.0f : ldx(c, k)) : in[c];
    const bool ii = i >= 1 && i <= im, jj = j >= 1 && j <= jm, kk = k >= 1 && k <= km;
    // what the forward sweep at swept cell x (plane d) took from this
    // location through coefficient coef
    auto from = [&](int x, int d, float coef) { return omega * (cn1[x] * coef) * ldx(x, d); };
    auto swept = [&](int a, int b, int d) { return ((a + b + d + nrd) & 1) != 0; };
    float r = v;
    if (ii && jj && kk) {
        if (swept(i, j, k)) {
            rhsb[c] -= (omega * cn1[c]) * v;
            r = (1.0f - omega) * v;
        } else {  // every interior neighbour was swept
            if (i > 1) r += from(nb(-1, 0, 0), k, g.cn2l[i - 1]);
            if (i < im) r += from(nb(1, 0, 0), k, g.cn2s[i + 1]);
            if (j > 1) r += from(nb(0, -1, 0), k, g.cn3l[j - 1]);
            if (j < jm) r += from(nb(0, 1, 0), k, g.cn3s[j + 1]);
            if (k > 1) r += from(nb(0, 0, -1), k - 1, g.cn4l[k - 1]);
            if (k < km) r += from(nb(0, 0, 1), k + 1, g.cn4s[k + 1]);
        }
    } else if (jj && kk && i == 0) {
        if (swept(1, j, k)) r += from(nb(1, 0, 0), k, g.cn2s[1]);
    } else if (jj && kk && i == im + 1) {
        if (swept(im, j, k)) r += from(nb(-1, 0, 0), k, g.cn2l[im]);
    } else if (ii && kk && j == 0) {
        if (swept(i, 1, k)) r += from(nb(0, 1, 0), k, g.cn3s[1]);
    } else if (ii && kk && j == jm + 1) {
        if (swept(i, jm, k)) r += from(nb(0, -1, 0), k, g.cn3l[jm]);
    } else if (ii && jj && k == 0) {
        if (swept(i, j, 1)) r += from(nb(0, 0, 1), 1, g.cn4s[1]);
    } else if (ii && jj && k == km + 1) {
        if (swept(i, j, km)) r += from(nb(0, 0, -1), km, g.cn4l[km]);
    }
    out[c] = r;
}

template <bool FOLDK>
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_sweep(Geo g, const float *in, float *out, float *rhsb,
                                                              const float *cn1, int nrd, float omega) {
    const int i = blockIdx.x * kAdjBX + threadIdx.x, j = blockIdx.y * kAdjBY + threadIdx.y, k = blockIdx.z;
    if (i > g.im + 2 || j > g.jm + 2) return;
    if (FOLDK && (k <= 2 || k >= g.km - 1))
        adj_sweep_cell<true>(g, in, out, rhsb, cn1, nrd, omega, i, j, k);
    else
        adj_sweep_cell<false>(g, in, out, rhsb, cn1, nrd, omega, i, j, k);
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
// With a force scale s (drag, f' = f + s fx) fx's adjoint is s times f's.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_feedbf(Geo g, Fields F, float *fxb, float *fyb, float *fzb,
                                                               float alpha, float dt, float beta,
                                                               const float *drag = nullptr) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    const float s = drag ? drag[(i - 1) + g.im * (j - 1)] : 1.0f;
    auto comp = [&](float *sumb, float *vb, const float *mask, float *xb, const float *fb) {
        const float m = mask[c];
        const float t = xb[c] + (drag ? s * fb[c] : fb[c]);
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

// ---- les.f95:31-182 (Smagorinsky sm, boundsm, viscous terms) ------------
// Nonlinear: the adjoint is taken at the forward state (the caller's diu and
// the sm they give).  Contributions are scattered with atomic adds, so the
// adjoint's last bits depend on the order the adds land in.
struct LesAdj {
    Geo g;
    const float *d[9];  // diu1..9 (forward values)
    float *db[9];       // their adjoints (accumulated)
    const float *sm;    // sm of the forward, boundsm included
    float *smb;         // sm's adjoint
};

// The viscous terms transposed (les.f95:170-274): f, g, h gain
// vf = sum sgn * evs * D / div per cell, evs a value of sm or a two-axis
// weighted average of four, D = 2 diu or the sum of two diu values; each
// term sends vb * D (vb = sgn * seed / div) to the sm points of evs, with
// their weights, and vb * evs to the diu entries of D.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_les_visc(LesAdj a, const float *fb, const float *gb,
                                                                 const float *hb) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    const Geo &g = a.g;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    const float sf = fb[c], sg = gb[c], sh = hb[c];
    auto X = [&](int q) { return g.dx1[q]; };
    auto Y = [&](int q) { return g.dy1[q]; };
    auto Z = [&](int q) { return g.dzn[q]; };
    auto S = [&](int x, int y, int z) { return a.sm[IX(g, x, y, z)]; };
    auto sadd = [&](int x, int y, int z, float v) { atomicAdd(&a.smb[IX(g, x, y, z)], v); };
    auto dv = [&](int n, int x, int y, int z) { return a.d[n][IX(g, x, y, z)]; };
    auto dadd = [&](int n, int x, int y, int z, float v) { atomicAdd(&a.db[n][IX(g, x, y, z)], v); };
    // evs = sm(px,py,pz), D = 2 diu_n(qx,qy,qz)
    auto pt = [&](float seed, float sgn, float div, int px, int py, int pz, int n, int qx, int qy, int qz) {
        const float vb = sgn * seed / div;
        sadd(px, py, pz, vb * (2.0f * dv(n, qx, qy, qz)));
        dadd(n, qx, qy, qz, vb * S(px, py, pz) * 2.0f);
    };
    // evs = (A*((d(p+1) s(p,q0) + d(p) s(p+1,q0))/Sin) + B*(... at q0+1))/Sd,
    // inner axis ax (0 x, 1 y) over p, p+1, outer axis bx (1 y, 2 z) over
    // q0, q0+1; D = diu_n1(..) + diu_n2(..)
    auto av = [&](float seed, float sgn, float div, int ax, int p, int bx, int q0, float A, float B, float Sd,
                  int n1, int x1, int y1, int z1, int n2, int x2, int y2, int z2) {
        const float dp = ax == 0 ? X(p) : Y(p), dp1 = ax == 0 ? X(p + 1) : Y(p + 1);
        const float Sin = dp + dp1;
        int px[4], py[4], pz[4];
        float w[4], evs = 0.0f;
#pragma unroll
        for (int o = 0; o < 2; ++o)
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int q = 2 * o + t;
                px[q] = i;
                py[q] = j;
                pz[q] = k;
                if (ax == 0) px[q] = p + t;
                else py[q] = p + t;
                if (bx == 1) py[q] = q0 + o;
                else pz[q] = q0 + o;
                w[q] = (o ? B : A) * (t ? dp : dp1) / Sin / Sd;
                evs += w[q] * S(px[q], py[q], pz[q]);
            }
        const float D = dv(n1, x1, y1, z1) + dv(n2, x2, y2, z2);
        const float vb = sgn * seed / div;
#pragma unroll
        for (int q = 0; q < 4; ++q) sadd(px[q], py[q], pz[q], vb * D * w[q]);
        dadd(n1, x1, y1, z1, vb * evs);
        dadd(n2, x2, y2, z2, vb * evs);
    };
    // f (les.f95:170-204)
    pt(sf, 1.0f, X(i), i + 1, j, k, 0, i + 1, j, k);
    pt(sf, -1.0f, X(i), i, j, k, 0, i, j, k);
    av(sf, 1.0f, Y(j), 0, i, 1, j, Y(j + 1), Y(j), Y(j) + Y(j + 1), 1, i, j + 1, k, 3, i + 1, j, k);
    av(sf, -1.0f, Y(j), 0, i, 1, j - 1, Y(j + 1), Y(j), Y(j) + Y(j + 1), 1, i, j, k, 3, i + 1, j - 1, k);
    av(sf, 1.0f, Z(k), 0, i, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 2, i, j, k + 1, 6, i + 1, j, k);
    av(sf, -1.0f, Z(k), 0, i, 2, k - 1, Z(k), Z(k - 1), Z(k - 1) + Z(k), 2, i, j, k, 6, i + 1, j, k - 1);
    // g (les.f95:205-239)
    av(sg, 1.0f, X(i), 0, i, 1, j, Y(j + 1), Y(j), Y(j) + Y(j + 1), 1, i, j + 1, k, 3, i + 1, j, k);
    av(sg, -1.0f, X(i), 0, i - 1, 1, j, Y(j + 1), Y(j), Y(j) + Y(j + 1), 1, i - 1, j + 1, k, 3, i, j, k);
    pt(sg, 1.0f, Y(j), i, j + 1, k, 4, i, j + 1, k);
    pt(sg, -1.0f, Y(j), i, j, k, 4, i, j, k);
    av(sg, 1.0f, Z(k), 0, i, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 5, i, j, k + 1, 7, i, j + 1, k);
    av(sg, -1.0f, Z(k), 0, i, 2, k - 1, Z(k), Z(k - 1), Z(k - 1) + Z(k), 5, i, j, k, 7, i, j + 1, k - 1);
    // h (les.f95:240-274)
    av(sh, 1.0f, X(i), 0, i, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 2, i, j, k + 1, 6, i + 1, j, k);
    av(sh, -1.0f, X(i), 0, i - 1, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 2, i - 1, j, k + 1, 6, i, j, k);
    av(sh, 1.0f, Y(j), 1, j, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 5, i, j, k + 1, 7, i, j + 1, k);
    av(sh, -1.0f, Y(j), 1, j - 1, 2, k, Z(k + 1), Z(k), Z(k) + Z(k + 1), 5, i, j - 1, k + 1, 7, i, j, k);
    pt(sh, 1.0f, Z(k), i, j, k + 1, 8, i, j, k + 1);
    pt(sh, -1.0f, Z(k), i, j, k, 8, i, j, k);
}

// boundsm transposed (boundsm.f95:13-32), its three loops last first:
// k ghosts sm(.,.,0) = -sm(.,.,1), sm(.,.,km+1) = sm(.,.,km) over
// j = -1..jm+1, i = 0..im+1 (stage 3); j ghosts sm(.,jm+1,.) = sm(.,jm,.),
// sm(.,0,.) = sm(.,1,.) over k = 0..km+1, i = 0..im+1 (stage 2); i ghosts
// sm(0,.,.) = sm(1,.,.), sm(im+1,.,.) = sm(im,.,.) over k = 0..km+1,
// j = -1..jm+1 (stage 1).
__global__ void k_adj_boundsm(Geo g, float *smb, int stage) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int im = g.im, jm = g.jm, km = g.km;
    auto at = [&](int x, int y, int z) -> float & { return smb[IX(g, x, y, z)]; };
    if (stage == 3) {
        const int ni = im + 2;
        if (t >= ni * (jm + 3)) return;
        const int i = t % ni, j = t / ni - 1;
        at(i, j, km) += at(i, j, km + 1);
        at(i, j, km + 1) = 0.0f;
        at(i, j, 1) += -at(i, j, 0);
        at(i, j, 0) = 0.0f;
    } else if (stage == 2) {
        const int ni = im + 2;
        if (t >= ni * (km + 2)) return;
        const int i = t % ni, k = t / ni;
        at(i, 1, k) += at(i, 0, k);
        at(i, 0, k) = 0.0f;
        at(i, jm, k) += at(i, jm + 1, k);
        at(i, jm + 1, k) = 0.0f;
    } else {
        const int nj = jm + 3;
        if (t >= nj * (km + 2)) return;
        const int j = t % nj - 1, k = t / nj;
        at(im, j, k) += at(im + 1, j, k);
        at(im + 1, j, k) = 0.0f;
        at(1, j, k) += at(0, j, k);
        at(0, j, k) = 0.0f;
    }
}

// sm = smc(k) sqrt(Q) transposed (les.f95:132-152), Q = 2(d1^2 + d5^2 +
// d9^2) + a^2 + b^2 + c^2 of the cell's averaged gradients; at Q = 0 (all
// gradients zero, e.g. inside buildings) sqrt has no derivative and none is
// propagated.  The forward overwrites sm here: its input adjoint is 0.
__global__ void __launch_bounds__(kAdjBX *kAdjBY) k_adj_les_sm(LesAdj a) {
    const int i = 1 + blockIdx.x * kAdjBX + threadIdx.x, j = 1 + blockIdx.y * kAdjBY + threadIdx.y;
    const int k = 1 + blockIdx.z;
    const Geo &g = a.g;
    if (i > g.im || j > g.jm) return;
    auto dv = [&](int n, int x, int y, int z) { return a.d[n][IX(g, x, y, z)]; };
    auto dadd = [&](int n, int x, int y, int z, float v) { atomicAdd(&a.db[n][IX(g, x, y, z)], v); };
    float &sb = a.smb[IX(g, i, j, k)];
    const float b0 = sb;
    sb = 0.0f;
    const float d1 = dv(0, i, j, k), d5 = dv(4, i, j, k), d9 = dv(8, i, j, k);
    const float uy = (dv(1, i - 1, j, k) + dv(1, i - 1, j + 1, k) + dv(1, i, j, k) + dv(1, i, j + 1, k)) * 0.25f;
    const float uz = (dv(2, i - 1, j, k) + dv(2, i - 1, j, k + 1) + dv(2, i, j, k) + dv(2, i, j, k + 1)) * 0.25f;
    const float vx = (dv(3, i, j, k) + dv(3, i, j - 1, k) + dv(3, i + 1, j, k) + dv(3, i + 1, j - 1, k)) * 0.25f;
    const float vz = (dv(5, i, j - 1, k) + dv(5, i, j - 1, k + 1) + dv(5, i, j, k) + dv(5, i, j, k + 1)) * 0.25f;
    const float wx = (dv(6, i, j, k) + dv(6, i, j, k - 1) + dv(6, i + 1, j, k) + dv(6, i + 1, j, k - 1)) * 0.25f;
    const float wy = (dv(7, i, j, k) + dv(7, i, j, k - 1) + dv(7, i, j + 1, k) + dv(7, i, j + 1, k - 1)) * 0.25f;
    const float ab = uy + vx, bb = wy + vz, cb = uz + wx;
    const float q = 2.0f * (d1 * d1 + d5 * d5 + d9 * d9) + ab * ab + bb * bb + cb * cb;
    if (!(q > 0.0f)) return;
    const float qb = b0 * g.smc[k] * 0.5f / sqrtf(q);
    dadd(0, i, j, k, qb * 4.0f * d1);
    dadd(4, i, j, k, qb * 4.0f * d5);
    dadd(8, i, j, k, qb * 4.0f * d9);
    const float a4 = 0.5f * ab * qb, b4 = 0.5f * bb * qb, c4 = 0.5f * cb * qb;  // 2 x * qb / 4
    dadd(1, i - 1, j, k, a4);
    dadd(1, i - 1, j + 1, k, a4);
    dadd(1, i, j, k, a4);
    dadd(1, i, j + 1, k, a4);
    dadd(3, i, j, k, a4);
    dadd(3, i, j - 1, k, a4);
    dadd(3, i + 1, j, k, a4);
    dadd(3, i + 1, j - 1, k, a4);
    dadd(2, i - 1, j, k, c4);
    dadd(2, i - 1, j, k + 1, c4);
    dadd(2, i, j, k, c4);
    dadd(2, i, j, k + 1, c4);
    dadd(6, i, j, k, c4);
    dadd(6, i, j, k - 1, c4);
    dadd(6, i + 1, j, k, c4);
    dadd(6, i + 1, j, k - 1, c4);
    dadd(5, i, j - 1, k, b4);
    dadd(5, i, j - 1, k + 1, b4);
    dadd(5, i, j, k, b4);
    dadd(5, i, j, k + 1, b4);
    dadd(7, i, j, k, b4);
    dadd(7, i, j, k - 1, b4);
    dadd(7, i, j + 1, k, b4);
    dadd(7, i, j + 1, k - 1, b4);
}

}  // namespace
}  // namespace les
