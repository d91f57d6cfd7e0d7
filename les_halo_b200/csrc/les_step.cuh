// les_step.cuh -- momentum part of the time step (velnw .. adam).
//
// One thread per interior cell unless a kernel says otherwise.  Every
// expression keeps the operand order of the reference's Fortran, and the
// library is compiled with --fmad=false, so results are bit-identical to a
// strict-IEEE evaluation of the reference.
#pragma once
#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

// velnw.f95:27-59 fused with the inflow of bondv1.f95:26-45 /
// bondv1_ext_wind_profile.f95:27-35 and the n==1 broadcast of
// bondv1.f95:47-59 (ICAL=0).  Cells i in 0..im, j in 1..jm, k in 1..km.
// VELNW=false gives the bondv1 part alone (ifdata.f95:258); INFLOW=false
// gives velnw alone (velnw.f95, the per-routine entry).
template <bool VELNW, bool INFLOW>
__device__ __forceinline__ void velnw_cell(const Geo &g, const Fields &F, int n, int ical, int i, int j, int k) {
    const int c = IX(g, i, j, k);
    const bool bc = INFLOW && ((i <= 1) || (n == 1 && ical == 0));
    if (bc) {
        F.u[c] = g.wind[(j - 1) + g.jm * (k - 1)];
        F.v[c] = 0.0f;
        F.w[c] = 0.0f;
        return;
    }
    if (!VELNW) return;
    // every load before the first store (the compiler cannot move loads
    // across stores to possibly aliasing fields)
    const bool wz = (k <= g.km - 1);
    const float pc = F.p[c], pe = F.p[IX(g, i + 1, j, k)], pn = F.p[IX(g, i, j + 1, k)];
    const float pu = wz ? F.p[IX(g, i, j, k + 1)] : 0.0f;
    const float uc = F.u[c], vc = F.v[c], wc = wz ? F.w[c] : 0.0f;
    const float fc = F.f[c], gc = F.g[c], hc = wz ? F.h[c] : 0.0f;
    {
        float pz = (-pc + pe) / g.ro / g.dxs[i];
        F.u[c] = uc + g.dt * (fc - pz);
    }
    {
        float pz = (-pc + pn) / g.ro / g.dys[j];
        F.v[c] = vc + g.dt * (gc - pz);
    }
    if (wz) {
        float pz = (-pc + pu) / g.ro / g.dzs[k];
        F.w[c] = wc + g.dt * (hc - pz);
    }
}

// Warps cover i = 1..im from the start of a 128-byte line (box offset 32);
// the i = 0 inflow column is done by lane 0 of the first block column.
template <bool VELNW, bool INFLOW = true>
__global__ void __launch_bounds__(128) k_velnw_inflow(Geo g, Fields F, int n, int ical) {
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (j > g.jm) return;
    const int i = 1 + blockIdx.x * 32 + threadIdx.x;
    if (i <= g.im) velnw_cell<VELNW, INFLOW>(g, F, n, ical, i, j, k);
    if (INFLOW && blockIdx.x == 0 && threadIdx.x == 0) velnw_cell<VELNW, INFLOW>(g, F, n, ical, 0, j, k);
}

// bondv1.f95:67-74: aaa = max(0, u(im,:,:)), bbb = min(0, u(im,:,:)).
// Positive floats order like their bit patterns, so integer atomicMax works.
__global__ void __launch_bounds__(256) k_uout_reduce(Geo g, const float *__restrict__ u, Scal *s) {
    unsigned int pos = 0u, neg = 0u;
    const int nface = g.jm * g.km;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nface; t += gridDim.x * blockDim.x) {
        const int j = 1 + t % g.jm, k = 1 + t / g.jm;
        const float x = u[IX(g, g.im, j, k)];
        if (x > 0.0f) pos = max(pos, __float_as_uint(x));
        if (x < 0.0f) neg = max(neg, __float_as_uint(-x));
    }
    for (int off = 16; off >= 1; off >>= 1) {
        pos = max(pos, __shfl_down_sync(0xffffffffu, pos, off));
        neg = max(neg, __shfl_down_sync(0xffffffffu, neg, off));
    }
    if ((threadIdx.x & 31) == 0) {
        if (pos) atomicMax(&s->uout_pos, pos);
        if (neg) atomicMax(&s->uout_neg, neg);
    }
}

// bondv1.f95:75-97: uout and the advective outflow on (j,k) in 1..jm x 1..km.
__global__ void __launch_bounds__(256) k_outflow(Geo g, Fields F, Scal *s) {
    const float aaa = __uint_as_float(s->uout_pos);
    const float bbb = s->uout_neg ? -__uint_as_float(s->uout_neg) : 0.0f;
    const float uout = (aaa + bbb) / 2.0f;
    const int nface = g.jm * g.km;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) s->uout = uout;
    if (t >= nface) return;
    const int j = 1 + t % g.jm, k = 1 + t / g.jm, im = g.im;
    const float rdx = g.dxs[im];
    {
        const int a = IX(g, im, j, k), b = IX(g, im - 1, j, k);
        F.u[a] = F.u[a] - g.dt * uout * (F.u[a] - F.u[b]) / rdx;
    }
    {
        const int a = IX(g, im + 1, j, k), b = IX(g, im, j, k);
        F.v[a] = F.v[a] - g.dt * uout * (F.v[a] - F.v[b]) / rdx;
        F.w[a] = F.w[a] - g.dt * uout * (F.w[a] - F.w[b]) / rdx;
    }
}

// bondv1.f95:99-137: periodic j rows, then top/ground planes, written as the
// final value each ghost holds (its source is always an interior row/plane
// that this kernel does not write).  The w loop of bondv1.f95:132-137 starts
// at i=-1, one below w's lower bound; in the reference's column-major layout
// that writes w(ip+1,j-1,0/km) (already zeroed by i=im+1) and, for j=-1,
// w(ip+1,jp+1,-1) and w(ip+1,jp+1,km-1).  Those two are zeroed here too.
__global__ void __launch_bounds__(256) k_uvw_ghosts(Geo g, Fields F) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int ni = im + 2;
    const int nA = 2 * km * ni;          // rows j=0,jm+1 ; k=1..km ; i=0..im+1
    const int nB = 2 * (jm + 2) * ni;    // u,v planes k=0,km+1 ; j=0..jm+1
    const int nC = 2 * (jm + 3) * ni;    // w planes k=0,km ; j=-1..jm+1
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nA) {
        const int i = t % ni;
        const int r = t / ni;
        const int k = 1 + r % km;
        const bool top = (r / km) != 0;
        const int j = top ? jm + 1 : 0, js = top ? 1 : jm;
        const int d = IX(g, i, j, k), s = IX(g, i, js, k);
        F.u[d] = F.u[s];
        F.v[d] = F.v[s];
        if (k <= km - 1) F.w[d] = (top && i == im + 1 && k == km - 1) ? 0.0f : F.w[s];
        return;
    }
    t -= nA;
    if (t < nB) {
        const int i = t % ni;
        const int r = t / ni;
        const int j = r % (jm + 2);
        const bool top = (r / (jm + 2)) != 0;
        const int js = (j == 0) ? jm : (j == jm + 1 ? 1 : j);
        if (!top) {
            const int d = IX(g, i, j, 0), s = IX(g, i, js, 1);
            F.u[d] = -F.u[s];
            F.v[d] = -F.v[s];
        } else {
            const int d = IX(g, i, j, km + 1), s = IX(g, i, js, km);
            F.u[d] = F.u[s];
            F.v[d] = F.v[s];
        }
        return;
    }
    t -= nB;
    if (t < nC) {
        const int i = t % ni;
        const int r = t / ni;
        const int j = -1 + r % (jm + 3);
        const int k = (r / (jm + 3)) ? km : 0;
        F.w[IX(g, i, j, k)] = 0.0f;
        if (i == im + 1 && j == jm + 1 && k == 0) F.w[IX(g, im + 1, jm + 1, -1)] = 0.0f;
    }
}

// Sources of the nine strain-rate arrays diu1..9 read by les.f95: computed
// on the fly from u,v,w (the fused step), or the caller's arrays held in
// box layout (the les per-routine entry, which receives diu as input).
struct DiuOnFly : DivIEEE {
    Geo g;
    UVW q;
    __device__ __forceinline__ float d1(int i, int j, int k) const { return diu1_e(g, q, i, j, k); }
    __device__ __forceinline__ float d2(int i, int j, int k) const { return diu2_e(g, q, i, j, k); }
    __device__ __forceinline__ float d3(int i, int j, int k) const { return diu3_e(g, q, i, j, k); }
    __device__ __forceinline__ float d4(int i, int j, int k) const { return diu4_e(g, q, i, j, k); }
    __device__ __forceinline__ float d5(int i, int j, int k) const { return diu5_e(g, q, i, j, k); }
    __device__ __forceinline__ float d6(int i, int j, int k) const { return diu6_e(g, q, i, j, k); }
    __device__ __forceinline__ float d7(int i, int j, int k) const { return diu7_e(g, q, i, j, k); }
    __device__ __forceinline__ float d8(int i, int j, int k) const { return diu8_e(g, q, i, j, k); }
    __device__ __forceinline__ float d9(int i, int j, int k) const { return diu9_e(g, q, i, j, k); }
};
struct DiuBoxes : DivIEEE {
    Geo g;
    const float *a[9];
    __device__ __forceinline__ float at(int n, int i, int j, int k) const { return __ldg(&a[n][IX(g, i, j, k)]); }
    __device__ __forceinline__ float d1(int i, int j, int k) const { return at(0, i, j, k); }
    __device__ __forceinline__ float d2(int i, int j, int k) const { return at(1, i, j, k); }
    __device__ __forceinline__ float d3(int i, int j, int k) const { return at(2, i, j, k); }
    __device__ __forceinline__ float d4(int i, int j, int k) const { return at(3, i, j, k); }
    __device__ __forceinline__ float d5(int i, int j, int k) const { return at(4, i, j, k); }
    __device__ __forceinline__ float d6(int i, int j, int k) const { return at(5, i, j, k); }
    __device__ __forceinline__ float d7(int i, int j, int k) const { return at(6, i, j, k); }
    __device__ __forceinline__ float d8(int i, int j, int k) const { return at(7, i, j, k); }
    __device__ __forceinline__ float d9(int i, int j, int k) const { return at(8, i, j, k); }
};

// velFG.f95:58-105 for one cell: f and g always, h when k <= km-1.  The
// dfu1/dfv1/dfw1 terms are returned too.
__device__ __forceinline__ void velfg_cell(const Geo &g, const UVW &q, int i, int j, int k, float &fv, float &gv,
                                           float &hv, float &dfu1, float &dfv1, float &dfw1) {
    const float *dx1 = g.dx1, *dy1 = g.dy1, *dzn = g.dzn, *dzs = g.dzs;
    {  // --u velocity, velFG.f95:59-72
        float covx1 = (dx1[i + 1] * cov1_e(g, q, i, j, k) + dx1[i] * cov1_e(g, q, i + 1, j, k)) /
                      (dx1[i] + dx1[i + 1]);
        float covy1 = (cov2_e(g, q, i, j, k) + cov2_e(g, q, i, j + 1, k)) / 2.0f;
        float covz1 = (cov3_e(g, q, i, j, k) + cov3_e(g, q, i, j, k + 1)) / 2.0f;
        float covc = covx1 + covy1 + covz1;
        dfu1 = 2.0f * (-diu1_e(g, q, i, j, k) + diu1_e(g, q, i + 1, j, k)) / (dx1[i] + dx1[i + 1]) +
               (-diu2_e(g, q, i, j, k) + diu2_e(g, q, i, j + 1, k)) / dy1[j] +
               (-diu3_e(g, q, i, j, k) + diu3_e(g, q, i, j, k + 1)) / dzn[k];
        float df = g.vn * dfu1;
        fv = (-covc + df);
    }
    {  // --v velocity, velFG.f95:75-88
        float covx1 = (cov4_e(g, q, i, j, k) + cov4_e(g, q, i + 1, j, k)) / 2.0f;
        float covy1 = (dy1[j + 1] * cov5_e(g, q, i, j, k) + dy1[j] * cov5_e(g, q, i, j + 1, k)) /
                      (dy1[j] + dy1[j + 1]);
        float covz1 = (cov6_e(g, q, i, j, k) + cov6_e(g, q, i, j, k + 1)) / 2.0f;
        float covc = covx1 + covy1 + covz1;
        dfv1 = (-diu4_e(g, q, i, j, k) + diu4_e(g, q, i + 1, j, k)) / dx1[i] +
               2.0f * (-diu5_e(g, q, i, j, k) + diu5_e(g, q, i, j + 1, k)) / (dy1[j] + dy1[j + 1]) +
               (-diu6_e(g, q, i, j, k) + diu6_e(g, q, i, j, k + 1)) / dzn[k];
        float df = g.vn * dfv1;
        gv = (-covc + df);
    }
    if (k <= g.km - 1) {  // --w velocity, velFG.f95:92-105
        float covx1 = (cov7_e(g, q, i, j, k) + cov7_e(g, q, i + 1, j, k)) / 2.0f;
        float covy1 = (cov8_e(g, q, i, j, k) + cov8_e(g, q, i, j + 1, k)) / 2.0f;
        float covz1 = (dzn[k + 1] * cov9_e(g, q, i, j, k) + dzn[k] * cov9_e(g, q, i, j, k + 1)) /
                      (dzn[k] + dzn[k + 1]);
        float covc = covx1 + covy1 + covz1;
        dfw1 = (-diu7_e(g, q, i, j, k) + diu7_e(g, q, i + 1, j, k)) / dx1[i] +
               (-diu8_e(g, q, i, j, k) + diu8_e(g, q, i, j + 1, k)) / dy1[j] +
               (-diu9_e(g, q, i, j, k) + diu9_e(g, q, i, j, k + 1)) / dzs[k];
        float df = g.vn * dfw1;
        hv = (-covc + df);
    }
}

// les.f95:132-150 sgs eddy viscosity at one interior cell.
template <class D>
__device__ __forceinline__ float sgs_sm(const Geo &g, const D &d, int i, int j, int k) {
    float dudxx1 = d.d1(i, j, k);
    float dudyx1 = (d.d2(i - 1, j, k) + d.d2(i - 1, j + 1, k) + d.d2(i, j, k) + d.d2(i, j + 1, k)) * 0.25f;
    float dudzx1 = (d.d3(i - 1, j, k) + d.d3(i - 1, j, k + 1) + d.d3(i, j, k) + d.d3(i, j, k + 1)) * 0.25f;
    float dvdxx1 = (d.d4(i, j, k) + d.d4(i, j - 1, k) + d.d4(i + 1, j, k) + d.d4(i + 1, j - 1, k)) * 0.25f;
    float dvdyx1 = d.d5(i, j, k);
    float dvdzx1 = (d.d6(i, j - 1, k) + d.d6(i, j - 1, k + 1) + d.d6(i, j, k) + d.d6(i, j, k + 1)) * 0.25f;
    float dwdxx1 = (d.d7(i, j, k) + d.d7(i, j, k - 1) + d.d7(i + 1, j, k) + d.d7(i + 1, j, k - 1)) * 0.25f;
    float dwdyx1 = (d.d8(i, j, k) + d.d8(i, j, k - 1) + d.d8(i, j + 1, k) + d.d8(i, j + 1, k - 1)) * 0.25f;
    float dwdzx1 = d.d9(i, j, k);
    float a = dudyx1 + dvdxx1, b = dwdyx1 + dvdzx1, cc = dudzx1 + dwdxx1;
    return g.smc[k] * sqrtf(2.0f * (dudxx1 * dudxx1 + dvdyx1 * dvdyx1 + dwdzx1 * dwdzx1) + a * a + b * b + cc * cc);
}

// les.f95:170-274 viscous flux divergence at one interior cell.
template <class D>
__device__ __forceinline__ void visc_cell(const Geo &g, const D &d, const float *__restrict__ sm, int i, int j, int k,
                                          float &vfu, float &vfv, float &vfw) {
    const float *dx1 = g.dx1, *dy1 = g.dy1, *dzn = g.dzn;
#define SM(a, b, c) __ldg(&sm[IX(g, (a), (b), (c))])
    {  // x-comp, les.f95:170-201
        float evsx2 = SM(i + 1, j, k);
        float evsx1 = SM(i, j, k);
        float evsy2 = d.xd((dy1[j + 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dy1[j] * (d.xd((dx1[i + 1] * SM(i, j + 1, k) + dx1[i] * SM(i + 1, j + 1, k)), dx1[i] + dx1[i + 1], g.rsx[i]))), dy1[j] + dy1[j + 1], g.rsy[j]);
        float evsy1 = d.xd((dy1[j + 1] * (d.xd((dx1[i + 1] * SM(i, j - 1, k) + dx1[i] * SM(i + 1, j - 1, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dy1[j] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i]))), dy1[j] + dy1[j + 1], g.rsy[j]);
        float evsz2 = d.zn2(g, (dzn[k + 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dzn[k] * (d.xd((dx1[i + 1] * SM(i, j, k + 1) + dx1[i] * SM(i + 1, j, k + 1)), dx1[i] + dx1[i + 1], g.rsx[i]))),
                      k);
        float evsz1 = d.zn2(g, (dzn[k] * (d.xd((dx1[i + 1] * SM(i, j, k - 1) + dx1[i] * SM(i + 1, j, k - 1)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dzn[k - 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i]))),
                      k - 1);
        float visux2 = (evsx2) * 2.0f * d.d1(i + 1, j, k);
        float visux1 = (evsx1) * 2.0f * d.d1(i, j, k);
        float visuy2 = (evsy2) * (d.d2(i, j + 1, k) + d.d4(i + 1, j, k));
        float visuy1 = (evsy1) * (d.d2(i, j, k) + d.d4(i + 1, j - 1, k));
        float visuz2 = (evsz2) * (d.d3(i, j, k + 1) + d.d7(i + 1, j, k));
        float visuz1 = (evsz1) * (d.d3(i, j, k) + d.d7(i + 1, j, k - 1));
        vfu = d.xd(visux2 - visux1, dx1[i], g.rdx1[i]) + d.xd(visuy2 - visuy1, dy1[j], g.rdy1[j]) + d.zn(g, visuz2 - visuz1, k);
    }
    {  // y-comp, les.f95:204-235
        float evsy2 = SM(i, j + 1, k);
        float evsy1 = SM(i, j, k);
        float evsx2 = d.xd((dy1[j + 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dy1[j] * (d.xd((dx1[i + 1] * SM(i, j + 1, k) + dx1[i] * SM(i + 1, j + 1, k)), dx1[i] + dx1[i + 1], g.rsx[i]))), dy1[j] + dy1[j + 1], g.rsy[j]);
        float evsx1 = d.xd((dy1[j + 1] * (d.xd((dx1[i] * SM(i - 1, j, k) + dx1[i - 1] * SM(i, j, k)), dx1[i - 1] + dx1[i], g.rsx[i - 1])) +
                       dy1[j] * (d.xd((dx1[i] * SM(i - 1, j + 1, k) + dx1[i - 1] * SM(i, j + 1, k)), dx1[i - 1] + dx1[i], g.rsx[i - 1]))), dy1[j] + dy1[j + 1], g.rsy[j]);
        float evsz2 = d.zn2(g, (dzn[k + 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dzn[k] * (d.xd((dx1[i + 1] * SM(i, j, k + 1) + dx1[i] * SM(i + 1, j, k + 1)), dx1[i] + dx1[i + 1], g.rsx[i]))),
                      k);
        float evsz1 = d.zn2(g, (dzn[k] * (d.xd((dx1[i + 1] * SM(i, j, k - 1) + dx1[i] * SM(i + 1, j, k - 1)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dzn[k - 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i]))),
                      k - 1);
        float visvx2 = (evsx2) * (d.d2(i, j + 1, k) + d.d4(i + 1, j, k));
        float visvx1 = (evsx1) * (d.d2(i - 1, j + 1, k) + d.d4(i, j, k));
        float visvy2 = (evsy2) * 2.0f * d.d5(i, j + 1, k);
        float visvy1 = (evsy1) * 2.0f * d.d5(i, j, k);
        float visvz2 = (evsz2) * (d.d6(i, j, k + 1) + d.d8(i, j + 1, k));
        float visvz1 = (evsz1) * (d.d6(i, j, k) + d.d8(i, j + 1, k - 1));
        vfv = d.xd(visvx2 - visvx1, dx1[i], g.rdx1[i]) + d.xd(visvy2 - visvy1, dy1[j], g.rdy1[j]) + d.zn(g, visvz2 - visvz1, k);
    }
    {  // z-comp, les.f95:238-272
        float evsz2 = SM(i, j, k + 1);
        float evsz1 = SM(i, j, k);
        float evsx2 = d.zn2(g, (dzn[k + 1] * (d.xd((dx1[i + 1] * SM(i, j, k) + dx1[i] * SM(i + 1, j, k)), dx1[i] + dx1[i + 1], g.rsx[i])) +
                       dzn[k] * (d.xd((dx1[i + 1] * SM(i, j, k + 1) + dx1[i] * SM(i + 1, j, k + 1)), dx1[i] + dx1[i + 1], g.rsx[i]))),
                      k);
        float evsx1 = d.zn2(g, (dzn[k + 1] * (d.xd((dx1[i] * SM(i - 1, j, k) + dx1[i - 1] * SM(i, j, k)), dx1[i - 1] + dx1[i], g.rsx[i - 1])) +
                       dzn[k] * (d.xd((dx1[i] * SM(i - 1, j, k + 1) + dx1[i - 1] * SM(i, j, k + 1)), dx1[i - 1] + dx1[i], g.rsx[i - 1]))),
                      k);
        float evsy2 = d.zn2(g, (dzn[k + 1] * (d.xd((dy1[j + 1] * SM(i, j, k) + dy1[j] * SM(i, j + 1, k)), dy1[j] + dy1[j + 1], g.rsy[j])) +
                       dzn[k] * (d.xd((dy1[j + 1] * SM(i, j, k + 1) + dy1[j] * SM(i, j + 1, k + 1)), dy1[j] + dy1[j + 1], g.rsy[j]))),
                      k);
        float evsy1 = d.zn2(g, (dzn[k + 1] * (d.xd((dy1[j] * SM(i, j - 1, k) + dy1[j - 1] * SM(i, j, k)), dy1[j - 1] + dy1[j], g.rsy[j - 1])) +
                       dzn[k] * (d.xd((dy1[j] * SM(i, j - 1, k + 1) + dy1[j - 1] * SM(i, j, k + 1)), dy1[j - 1] + dy1[j], g.rsy[j - 1]))),
                      k);
        float viswx2 = (evsx2) * (d.d3(i, j, k + 1) + d.d7(i + 1, j, k));
        float viswx1 = (evsx1) * (d.d3(i - 1, j, k + 1) + d.d7(i, j, k));
        float viswy2 = (evsy2) * (d.d6(i, j, k + 1) + d.d8(i, j + 1, k));
        float viswy1 = (evsy1) * (d.d6(i, j - 1, k + 1) + d.d8(i, j, k));
        float viswz2 = (evsz2) * 2.0f * d.d9(i, j, k + 1);
        float viswz1 = (evsz1) * 2.0f * d.d9(i, j, k);
        vfw = d.xd(viswx2 - viswx1, dx1[i], g.rdx1[i]) + d.xd(viswy2 - viswy1, dy1[j], g.rdy1[j]) + d.zn(g, viswz2 - viswz1, k);
    }
#undef SM
}

// feedbf.f95:38-66 for one cell: updates usum/vsum/wsum, returns fx,fy,fz.
__device__ __forceinline__ void feedbf_cell(const Geo &g, Fields &F, int c, float uc, float vc, float wc, float &fx,
                                            float &fy, float &fz) {
    const float bm = F.bmask[c], cm = F.cmask[c], dm = F.dmask[c];
    const float us = (F.usum[c] + uc) * bm;
    const float vs = (F.vsum[c] + vc) * cm;
    const float ws = (F.wsum[c] + wc) * dm;
    F.usum[c] = us;
    F.vsum[c] = vs;
    F.wsum[c] = ws;
    float f1x = g.alpha * us * g.dt, f1y = g.alpha * vs * g.dt, f1z = g.alpha * ws * g.dt;
    float f2x = g.beta * uc * bm, f2y = g.beta * vc * cm, f2z = g.beta * wc * dm;
    fx = f1x + f2x;
    fy = f1y + f2y;
    fz = f1z + f2z;
}

// boundsm.f95:13-32 as final values: ghost (i,j,k) = sign * sm(ci, cj, ck)
// with ci/cj/ck clamping 0->1 and im+1->im (jm, km alike) and sign -1 on
// the k=0 plane.  The j=-1 row keeps the values only the i-copy reaches.
// Every source is an interior cell or a j=-1 cell, neither of which this
// kernel writes.
__global__ void __launch_bounds__(256) k_boundsm(Geo g, float *__restrict__ sm) {
    const int im = g.im, jm = g.jm, km = g.km;
    const int nI = 2 * (jm + 3) * (km + 2);  // i = 0, im+1 ; j=-1..jm+1 ; k=0..km+1
    const int nJ = 2 * im * (km + 2);        // j = 0, jm+1 ; i=1..im ; k=0..km+1
    const int nK = 2 * im * (jm + 1);        // k = 0, km+1 ; i=1..im ; j=-1 and 1..jm
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t < nI) {
        i = (t & 1) ? im + 1 : 0;
        const int r = t >> 1;
        j = -1 + r % (jm + 3);
        k = r / (jm + 3);
    } else if ((t -= nI) < nJ) {
        j = (t & 1) ? jm + 1 : 0;
        const int r = t >> 1;
        i = 1 + r % im;
        k = r / im;
    } else if ((t -= nJ) < nK) {
        k = (t & 1) ? km + 1 : 0;
        const int r = t >> 1;
        i = 1 + r % im;
        const int jj = r / im;  // 0..jm : j = -1, 1..jm
        j = (jj == 0) ? -1 : jj;
    } else {
        return;
    }
    const int ci = i < 1 ? 1 : (i > im ? im : i);
    const int cj = (j == 0) ? 1 : (j == jm + 1 ? jm : j);
    const int ck = k < 1 ? 1 : (k > km ? km : k);
    const float s = sm[IX(g, ci, cj, ck)];
    sm[IX(g, i, j, k)] = (k == 0) ? -s : s;
}

// ifdata.f95:117-125 zero_arrays for f,g,h on (0:ip,0:jp,0:kp).
__global__ void k_zero_fgh(Geo g, Fields F) {
    const int n = (g.im + 1) * (g.jm + 1) * (g.km + 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t % (g.im + 1), r = t / (g.im + 1);
        const int j = r % (g.jm + 1), k = r / (g.jm + 1);
        const int c = IX(g, i, j, k);
        F.f[c] = 0.0f;
        F.g[c] = 0.0f;
        F.h[c] = 0.0f;
    }
}

}  // namespace
}  // namespace les
