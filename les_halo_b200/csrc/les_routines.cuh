// les_routines.cuh -- kernels of the per-routine drop-in entries
// (les_velnw_, les_velfg_, ...).  The whole-step path fuses these routines;
// the per-routine entries run them one at a time on caller arrays, so every
// element a reference routine does not write keeps the caller's value.
#pragma once
#include "les_step.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

// velFG.f95:58-105 alone: f, g (k<=km), h (k<=km-1) and, when the boxes are
// given, dfu1, dfv1 (k<=km) and dfw1 (k<=km-1).
__global__ void __launch_bounds__(128) k_velfg_only(Geo g, Fields F, float *dfu, float *dfv, float *dfw) {
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const UVW q{{}, F.u, F.v, F.w};
    const int c = IX(g, i, j, k);
    float fv, gv, hv = 0.0f, d1, d2, d3 = 0.0f;
    velfg_cell(g, q, i, j, k, fv, gv, hv, d1, d2, d3);
    F.f[c] = fv;
    F.g[c] = gv;
    if (k <= g.km - 1) F.h[c] = hv;
    if (dfu) dfu[c] = d1;
    if (dfv) dfv[c] = d2;
    if (dfw && k <= g.km - 1) dfw[c] = d3;
}

// vel2.f95:48-188: where the value of array `which` at (i,j,k) comes from.
// which = kind*9 + (n-1) with kind 0: nou, 1: diu, 2: cov and n = 1..9.
// Returns 1 (computed at (ci,cj,ck)), 2 (copied from a position vel2 never
// writes: the caller's value at (ci,cj,ck)) or 0 (not written).
__device__ __forceinline__ int vel2_source(const Geo &g, int which, int i, int j, int k, int &ci, int &cj, int &ck) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int n = which % 9 + 1, kind = which / 9;
    const bool diu = kind == 1;
    auto in = [](int x, int a, int b) { return x >= a && x <= b; };
    ci = i, cj = j, ck = k;
    int kmax = km;  // last computed k of the group
    if (n == 3 || n == 6) kmax = km + 1;
    if (n == 7 || n == 8) kmax = km - 1;
    // computed range
    if (in(i, 1, im) && in(j, 1, jm) && in(k, 1, kmax)) return 1;
    switch (n) {
        case 1: case 4: case 7:  // X(im+1,j,k) = X(im,j,k), j 1..jm, k 1..kmax
            if (i == im + 1 && in(j, 1, jm) && in(k, 1, kmax)) {
                ci = im;
                return 1;
            }
            break;
        case 2: case 5: case 8:  // X(i,0,k)=X(i,jm,k), X(i,jm+1,k)=X(i,1,k), i 1..im, k 1..kmax
            if (in(i, 1, im) && in(k, 1, kmax) && (j == 0 || j == jm + 1)) {
                cj = (j == 0) ? jm : 1;
                return 1;
            }
            break;
        default: break;
    }
    if (diu && (n == 2 || n == 3) && i == im + 1 && in(j, 1, jm + 1) && in(k, 1, km + 1)) {
        // diu2/diu3(im+1,j,k) = (im,j,k) for j 1..jm+1, k 1..km+1 (vel2.f95:177-182)
        ci = im;
        if (n == 2) {
            if (k <= km) {
                if (j == jm + 1) cj = 1;
                return 1;
            }
            return 2;
        }
        return (j <= jm) ? 1 : 2;
    }
    if (diu && (n == 4 || n == 6) && j == 0 && in(i, 1, im + 1) && in(k, 1, km + 1)) {
        // diu4/diu6(i,0,k) = (i,jm,k) for i 1..im+1, k 1..km+1 (vel2.f95:183-188)
        cj = jm;
        if (n == 4) {
            if (k <= km) {
                if (i == im + 1) ci = im;
                return 1;
            }
            return 2;
        }
        return (i <= im) ? 1 : 2;
    }
    return 0;
}

__device__ __forceinline__ float vel2_raw(const Geo &g, const UVW &q, int which, int i, int j, int k) {
    const int n = which % 9 + 1, kind = which / 9;
    float nou = 0.0f, diu = 0.0f;
    switch (n) {
        case 1: nou = nou1_raw(g, q, i, j, k); diu = diu1_raw(g, q, i, j, k); break;
        case 2: nou = nou2_raw(g, q, i, j, k); diu = diu2_raw(g, q, i, j, k); break;
        case 3: nou = nou3_raw(g, q, i, j, k); diu = diu3_raw(g, q, i, j, k); break;
        case 4: nou = nou4_raw(g, q, i, j, k); diu = diu4_raw(g, q, i, j, k); break;
        case 5: nou = nou5_raw(g, q, i, j, k); diu = diu5_raw(g, q, i, j, k); break;
        case 6: nou = nou6_raw(g, q, i, j, k); diu = diu6_raw(g, q, i, j, k); break;
        case 7: nou = nou7_raw(g, q, i, j, k); diu = diu7_raw(g, q, i, j, k); break;
        case 8: nou = nou8_raw(g, q, i, j, k); diu = diu8_raw(g, q, i, j, k); break;
        default: nou = nou9_raw(g, q, i, j, k); diu = diu9_raw(g, q, i, j, k); break;
    }
    if (kind == 0) return nou;
    if (kind == 1) return diu;
    return (n == 4 || n == 7) ? (nou - 0.0f) * diu : nou * diu;  // cov4/cov7: (nou - u0)*diu
}

// Write array `which` over its Fortran bounds li..ui x 0..jp+2 x 0..kp+2.
__global__ void k_vel2_out(Geo g, UVW q, float *box, int which, int li) {
    const int ni = g.im + 3 - li, nj = g.jm + 3, nk = g.km + 3;
    const long long n = (long long)ni * nj * nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = li + (int)(t % ni);
        const long long r = t / ni;
        const int j = (int)(r % nj), k = (int)(r / nj);
        int ci, cj, ck;
        const int src = vel2_source(g, which, i, j, k, ci, cj, ck);
        if (src == 1)
            box[IX(g, i, j, k)] = vel2_raw(g, q, which, ci, cj, ck);
        else if (src == 2)
            box[IX(g, i, j, k)] = box[IX(g, ci, cj, ck)];
    }
}

// feedbf.f95:38-67 alone; fx/fy/fz boxes optional.
__global__ void __launch_bounds__(128) k_feedbf_only(Geo g, Fields F, float *fxb, float *fyb, float *fzb) {
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    float fx, fy, fz;
    feedbf_cell(g, F, c, F.u[c], F.v[c], F.w[c], fx, fy, fz);
    if (fxb) fxb[c] = fx;
    if (fyb) fyb[c] = fy;
    if (fzb) fzb[c] = fz;
    F.f[c] = F.f[c] + fx;
    F.g[c] = F.g[c] + fy;
    F.h[c] = F.h[c] + fz;
}

// les.f95:132-152 from the caller's diu arrays.
__global__ void __launch_bounds__(128) k_les_sm(Geo g, DiuBoxes d, float *sm) {
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    sm[IX(g, i, j, k)] = sgs_sm(g, d, i, j, k);
}

// les.f95:170-274 from the caller's diu arrays (no adam).
__global__ void __launch_bounds__(128) k_les_visc(Geo g, DiuBoxes d, Fields F) {
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    float vfu, vfv, vfw;
    visc_cell(g, d, F.sm, i, j, k, vfu, vfv, vfw);
    const int c = IX(g, i, j, k);
    F.f[c] = F.f[c] + vfu;
    F.g[c] = F.g[c] + vfv;
    F.h[c] = F.h[c] + vfw;
}

// adam.f95:32-46 alone.
__global__ void __launch_bounds__(128) k_adam_only(Geo g, Fields F) {
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.im || j > g.jm) return;
    const int c = IX(g, i, j, k);
    const float fd = F.f[c], gd = F.g[c], hd = F.h[c];
    F.f[c] = 1.5f * fd - 0.5f * F.fold[c];
    F.g[c] = 1.5f * gd - 0.5f * F.gold[c];
    F.h[c] = 1.5f * hd - 0.5f * F.hold[c];
    F.fold[c] = fd;
    F.gold[c] = gd;
    F.hold[c] = hd;
}

// bondFG.f95:15-31 alone, one thread per (i,j,k) of the union of its loops.
__global__ void k_bondfg(Geo g, Fields F) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int nF = jm * km, nG = im * km, nH = 2 * im * jm;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nF) {
        const int j = 1 + t % jm, k = 1 + t / jm;
        F.f[IX(g, 0, j, k)] = F.f[IX(g, 1, j, k)];
    } else if ((t -= nF) < nG) {
        const int i = 1 + t % im, k = 1 + t / im;
        F.g[IX(g, i, 0, k)] = F.g[IX(g, i, jm, k)];
    } else if ((t -= nG) < nH) {
        const int i = 1 + t % im, r = t / im;
        const int j = 1 + r % jm;
        F.h[IX(g, i, j, (r / jm) ? km : 0)] = 0.0f;
    }
}

}  // namespace
}  // namespace les
