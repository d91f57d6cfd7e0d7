// les_halo.cuh -- halo ring pack/unpack (halo_exchange.cl) and the
// Fortran-layout <-> box repacking used at the host boundary.
//
// The reference launches one work-item per (k, i) pair and loops over the
// component and the ring width (halo_exchange.cl:3-291).  Here one thread
// owns one buffer element, so the buffer side is read or written fully
// coalesced; the array side is a gather/scatter along rows of the ring.
// Buffer layout per component v (stride v_sz): north | south | west | east.
#pragma once
#include "les_dev.cuh"

namespace les {
namespace {  // kernels get internal linkage: each .cu has its own copy

struct HaloDims {
    unsigned im, jm, km, hw, vdim;
    size_t vsz;     // floats per component
    size_t ns_sec;  // floats in the north (= south) section
    size_t we_sec;  // floats in the west (= east) section
};

__host__ __device__ inline HaloDims halo_dims(unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim,
                                              int inner) {
    HaloDims d;
    d.im = im;
    d.jm = jm;
    d.km = km;
    d.hw = hw;
    d.vdim = vdim;
    d.ns_sec = (size_t)km * (inner ? (im - 2 * hw) : im) * hw;
    d.we_sec = (size_t)km * (jm - 2 * hw) * hw;
    d.vsz = 2 * d.ns_sec + 2 * d.we_sec;
    return d;
}

// Array point index (i fastest, extents im x jm x km) of buffer offset o of
// one component.  Standard ring (halo_exchange.cl) or the owned inner ring
// (halo_exchange_correct.cl read).
__device__ __forceinline__ size_t halo_point(const HaloDims &d, size_t o, int inner) {
    const size_t im = d.im, jm = d.jm, hw = d.hw;
    if (o < 2 * d.ns_sec) {
        const bool south = o >= d.ns_sec;
        const size_t q = south ? o - d.ns_sec : o;
        const size_t rowlen = inner ? im - 2 * hw : im;
        const size_t i = q % rowlen, w = (q / rowlen) % hw, k = q / (rowlen * hw);
        if (!inner)
            return i + im * w + k * im * jm + (south ? im * (jm - hw) : 0);
        return south ? (i + hw) + k * im * jm + im * (jm - 2 * hw) + im * w : im * hw + (i + hw) + im * w + k * im * jm;
    }
    o -= 2 * d.ns_sec;
    const bool east = o >= d.we_sec;
    const size_t q = east ? o - d.we_sec : o;
    const size_t w = q % hw, r = (q / hw) % (jm - 2 * hw), k = q / ((jm - 2 * hw) * hw);
    const size_t row = (r + hw) * im + k * im * jm;
    if (!inner) return row + w + (east ? im - hw : 0);
    return row + w + (east ? im - 2 * hw : hw);
}

// exchange_N_halo_read (inner=0) / halo_exchange_correct.cl read (inner=1)
__global__ void k_halo_pack(const float *__restrict__ a, float *__restrict__ buf, HaloDims d, int inner) {
    const size_t total = d.vsz * d.vdim;
    for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < total; b += (size_t)gridDim.x * blockDim.x) {
        const size_t v = b / d.vsz, o = b % d.vsz;
        buf[b] = a[halo_point(d, o, inner) * d.vdim + v];
    }
}

// exchange_N_halo_write (inner=0).  The halo_exchange_correct.cl write
// (inner=1) reads the north/south buffer without the im*w row term, so all
// ring rows w take row 0's entries.
__global__ void k_halo_unpack(float *__restrict__ a, const float *__restrict__ buf, HaloDims d, int inner) {
    const size_t total = d.vsz * d.vdim;
    for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < total; b += (size_t)gridDim.x * blockDim.x) {
        const size_t v = b / d.vsz, o = b % d.vsz;
        size_t src = b;
        if (inner && o < 2 * d.ns_sec) {
            const bool south = o >= d.ns_sec;
            const size_t q = south ? o - d.ns_sec : o;
            const size_t i = q % d.im, k = q / ((size_t)d.im * d.hw);
            src = v * d.vsz + (south ? d.ns_sec : 0) + i + k * (size_t)d.im * d.hw;
        }
        a[halo_point(d, o, 0) * d.vdim + v] = buf[src];
    }
}

// Fortran array (bounds li..li+ni-1, lj.., lk..) <-> box.
__global__ void k_f2box(Geo g, float *__restrict__ box, const float *__restrict__ src, int li, int lj, int lk, int ni,
                        int nj, int nk) {
    const size_t n = (size_t)ni * nj * nk;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % ni), r = (int)(t / ni);
        const int j = r % nj, k = r / nj;
        box[IX(g, li + i, lj + j, lk + k)] = src[t];
    }
}
__global__ void k_box2f(Geo g, const float *__restrict__ box, float *__restrict__ dst, int li, int lj, int lk, int ni,
                        int nj, int nk, float sub, int sub_interior) {
    const size_t n = (size_t)ni * nj * nk;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int i = li + (int)(t % ni), r = (int)(t / ni);
        const int j = lj + r % nj, k = lk + r / nj;
        float x = box[IX(g, i, j, k)];
        if (sub_interior && i >= 1 && i <= g.im && j >= 1 && j <= g.jm && k >= 1 && k <= g.km) x = x - sub;
        dst[t] = x;
    }
}

// Context halo: pack/unpack the ring of a virtual AoS array whose
// components are box fields (NULL component -> 0 on read, ignored on write).
// Point (ii,jj,kk) of the combined array is Fortran (ii+li, jj+lj, kk+lk);
// component c exists only for k >= klo[c] (uvw's u,v start at k=0).
struct CombView {
    float *comp[4];
    int klo[4];
    int li, lj, lk;
};
__global__ void k_ctx_halo(Geo g, CombView cv, float *__restrict__ buf, HaloDims d, int write) {
    const size_t total = d.vsz * d.vdim;
    for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < total; b += (size_t)gridDim.x * blockDim.x) {
        const size_t v = b / d.vsz, o = b % d.vsz;
        const size_t pt = halo_point(d, o, 0);
        const int ii = (int)(pt % d.im), rr = (int)(pt / d.im);
        const int jj = rr % (int)d.jm, kk = rr / (int)d.jm;
        const int i = ii + cv.li, j = jj + cv.lj, k = kk + cv.lk;
        float *f = cv.comp[v];
        const bool ok = f != nullptr && k >= cv.klo[v];
        if (write) {
            if (ok) f[IX(g, i, j, k)] = buf[b];
        } else {
            buf[b] = ok ? f[IX(g, i, j, k)] : 0.0f;
        }
    }
}

}  // namespace
}  // namespace les
