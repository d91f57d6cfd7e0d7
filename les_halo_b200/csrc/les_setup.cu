// les_setup.cu -- setup routines feeding the step (grid metrics, Poisson
// coefficients, building masks), the halo entry points, and the seeded
// synthetic inputs of les_synth.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "les_abi.h"
#include "les_halo.cuh"
#include "les_synth.h"
#include "les_synth_gen.h"
#include "les_nvtx.h"

using namespace les;

// Error channel shared with les_lib.cu.
les_status les_internal_fail(les_status s, const char *msg);
les_status les_internal_ok();

namespace setup_impl {

#define CKS(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) return les_internal_fail(LES_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

// init.f95:82-107 on the device.
__global__ void k_poisson(int ip, int jp, int kp, const float *__restrict__ dxs, const float *__restrict__ dys,
                          const float *__restrict__ dzs_m1, float *cn1, float *cn2l, float *cn2s, float *cn3l,
                          float *cn3s, float *cn4l, float *cn4s) {
    const long long n = (long long)ip * jp * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(t % ip);
        const long long r = t / ip;
        const int j = 1 + (int)(r % jp), k = 1 + (int)(r / jp);
        const float dz1 = dzs_m1[k - 1 + 1], dz2 = dzs_m1[k + 1];
        const float c = 2.0f / (dxs[i - 1] * dxs[i]) + 2.0f / (dys[j - 1] * dys[j]) + 2.0f / (dz1 * dz2);
        cn1[t] = 1.0f / c;
        if (j == 1 && k == 1) {
            cn2s[i - 1] = 2.0f / (dxs[i - 1] * (dxs[i - 1] + dxs[i]));
            cn2l[i - 1] = 2.0f / (dxs[i] * (dxs[i - 1] + dxs[i]));
        }
        if (i == 1 && k == 1) {
            cn3s[j - 1] = 2.0f / (dys[j - 1] * (dys[j - 1] + dys[j]));
            cn3l[j - 1] = 2.0f / (dys[j] * (dys[j - 1] + dys[j]));
        }
        if (i == 1 && j == 1) {
            cn4s[k - 1] = 2.0f / (dz1 * (dz1 + dz2));
            cn4l[k - 1] = 2.0f / (dz2 * (dz1 + dz2));
        }
    }
}

// feedbfm.f95:42-62 on the device: interior (i,j,k) of the masks.
__global__ void k_masks(int ip, int jp, int kp, const float *__restrict__ zbm, const float *__restrict__ z2,
                        const float *__restrict__ dzn_m1, float *am, float *bm, float *cm, float *dm) {
    const long long n = (long long)ip * jp * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(t % ip);
        const long long r = t / ip;
        const int j = 1 + (int)(r % jp), k = 1 + (int)(r / jp);
        const float zb = zbm[(size_t)(i + 1) + (size_t)(ip + 3) * (j + 1)];
        const bool solid = zb > z2[k - 1] + 0.5f * dzn_m1[k + 1];
        const float a = solid ? 0.0f : 1.0f;
        const float o = (a == 0.0f) ? 1.0f : 0.0f;
        // amask1, dmask1: (0:ip+1,0:jp+1,0:kp+1); bmask1 (-1:ip+1,0:jp+1,0:kp+1); cmask1 (0:ip+1,-1:jp+1,0:kp+1)
        am[(size_t)i + (size_t)(ip + 2) * (j + (size_t)(jp + 2) * k)] = a;
        dm[(size_t)i + (size_t)(ip + 2) * (j + (size_t)(jp + 2) * k)] = o;
        bm[(size_t)(i + 1) + (size_t)(ip + 3) * (j + (size_t)(jp + 2) * k)] = o;
        cm[(size_t)i + (size_t)(ip + 2) * ((j + 1) + (size_t)(jp + 3) * k)] = o;
    }
}

les_status halo_common(const float *in, float *out, unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim,
                       int device, void *stream, int inner, int unpack) {
    if (!in || !out) return les_internal_fail(LES_ERR_BAD_ARG, "NULL array or buffer");
    if (!(vdim == 1 || vdim == 2 || vdim == 4 || vdim == 16))
        return les_internal_fail(LES_ERR_BAD_ARG, "vdim must be 1, 2, 4 or 16");
    if (hw == 0 || jm < 2 * hw || im < hw || km == 0 || (inner && im < 2 * hw))
        return les_internal_fail(LES_ERR_DIMS, "ring width does not fit the array");
    // the unpack of both variants uses the standard buffer layout
    const HaloDims d = halo_dims(im, jm, km, hw, vdim, unpack ? 0 : inner);
    const size_t nbuf = d.vsz * vdim, narr = (size_t)im * jm * km * vdim;
    cudaStream_t st = (cudaStream_t)stream;
    const float *a_in = in;
    float *a_out = out;
    DevBuf da, db;
    if (!device) {
        CKS(cudaMalloc(&da.p, sizeof(float) * narr));
        CKS(cudaMalloc(&db.p, sizeof(float) * nbuf));
        if (!unpack) {
            CKS(cudaMemcpyAsync(da.p, in, sizeof(float) * narr, cudaMemcpyHostToDevice, st));
            a_in = (const float *)da.p;
            a_out = (float *)db.p;
        } else {
            CKS(cudaMemcpyAsync(da.p, out, sizeof(float) * narr, cudaMemcpyHostToDevice, st));
            CKS(cudaMemcpyAsync(db.p, in, sizeof(float) * nbuf, cudaMemcpyHostToDevice, st));
            a_in = (const float *)db.p;
            a_out = (float *)da.p;
        }
    }
    const int blocks = (int)std::min<size_t>((nbuf + 255) / 256, 148 * 16);
    if (!unpack)
        k_halo_pack<<<blocks, 256, 0, st>>>(a_in, a_out, d, inner);
    else
        k_halo_unpack<<<blocks, 256, 0, st>>>(a_out, a_in, d, inner);
    CKS(cudaGetLastError());
    if (!device) {
        if (!unpack)
            CKS(cudaMemcpyAsync(out, db.p, sizeof(float) * nbuf, cudaMemcpyDeviceToHost, st));
        else
            CKS(cudaMemcpyAsync(out, da.p, sizeof(float) * narr, cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
    }
    return les_internal_ok();
}


}  // namespace setup_impl

using namespace setup_impl;

extern "C" {

les_status les_grid_metrics(int ip, int jp, int kp, float *dx1_, float *dxl_, float *dy1_, float *dyl_, float *z2_,
                            float *dzn_, float *dzs_, float *dxs_, float *dys_) {
    LES_RANGE("les_grid_metrics");
    if (!dx1_ || !dxl_ || !dy1_ || !dyl_ || !z2_ || !dzn_ || !dzs_ || !dxs_ || !dys_)
        return les_internal_fail(LES_ERR_BAD_ARG, "NULL array");
    auto dx1 = [&](int i) -> float & { return dx1_[i + 1]; };
    auto dy1 = [&](int j) -> float & { return dy1_[j]; };
    auto dzn = [&](int k) -> float & { return dzn_[k + 1]; };
    auto dzs = [&](int k) -> float & { return dzs_[k + 1]; };
    auto z2 = [&](int k) -> float & { return z2_[k - 1]; };
    // grid.f95:36-40, 49-51, 55-82
    dxl_[0] = 0.0f;
    for (int i = 1; i <= ip; ++i) dxl_[i] = dxl_[i - 1] + dx1(i);
    dyl_[0] = 0.0f;
    for (int j = 1; j <= jp; ++j) dyl_[j] = dyl_[j - 1] + dy1(j);
    z2(1) = dzn(1);
    dzn(kp + 2) = 0.0f;
    for (int k = 2; k <= kp + 2; ++k) z2(k) = z2(k - 1) + dzn(k);
    dzn(kp + 1) = dzn(kp);
    dzn(kp + 2) = dzn(kp + 1);
    dzn(0) = dzn(1);
    dzn(-1) = dzn(0);
    for (int k = 0; k <= kp; ++k) dzs(k) = dzn(k + 1) / 2.0f + dzn(k) / 2.0f;
    for (int i = 0; i <= ip; ++i) dxs_[i] = dx1(i) / 2.0f + dx1(i + 1) / 2.0f;
    for (int j = 0; j <= jp; ++j) dys_[j] = dy1(j) / 2.0f + dy1(j + 1) / 2.0f;
    dzs(kp + 1) = dzs(kp);
    dzs(kp + 2) = dzs(kp + 1);
    dzs(-1) = dzs(0);
    return les_internal_ok();
}

les_status les_poisson_coeffs(int ip, int jp, int kp, const float *dxs, const float *dys, const float *dzs,
                              float *cn1, float *cn2l, float *cn2s, float *cn3l, float *cn3s, float *cn4l,
                              float *cn4s) {
    LES_RANGE("les_poisson_coeffs");
    if (!dxs || !dys || !dzs || !cn1 || !cn2l || !cn2s || !cn3l || !cn3s || !cn4l || !cn4s)
        return les_internal_fail(LES_ERR_BAD_ARG, "NULL array");
    if (ip < 1 || jp < 1 || kp < 1) return les_internal_fail(LES_ERR_DIMS, "bad extents");
    const size_t n = (size_t)ip * jp * kp;
    DevBuf d_in, d_out;
    const size_t nin = (ip + 1) + (jp + 1) + (kp + 4);
    const size_t nout = n + 2 * (size_t)(ip + jp + kp);
    CKS(cudaMalloc(&d_in.p, sizeof(float) * nin));
    CKS(cudaMalloc(&d_out.p, sizeof(float) * nout));
    float *di = (float *)d_in.p, *dout = (float *)d_out.p;
    CKS(cudaMemcpy(di, dxs, sizeof(float) * (ip + 1), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(di + ip + 1, dys, sizeof(float) * (jp + 1), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(di + ip + 1 + jp + 1, dzs, sizeof(float) * (kp + 4), cudaMemcpyHostToDevice));
    float *o2l = dout + n, *o2s = o2l + ip, *o3l = o2s + ip, *o3s = o3l + jp, *o4l = o3s + jp, *o4s = o4l + kp;
    k_poisson<<<(int)std::min<size_t>((n + 255) / 256, 148 * 32), 256>>>(ip, jp, kp, di, di + ip + 1, di + ip + jp + 2,
                                                                          dout, o2l, o2s, o3l, o3s, o4l, o4s);
    CKS(cudaGetLastError());
    CKS(cudaMemcpy(cn1, dout, sizeof(float) * n, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn2l, o2l, sizeof(float) * ip, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn2s, o2s, sizeof(float) * ip, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn3l, o3l, sizeof(float) * jp, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn3s, o3s, sizeof(float) * jp, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn4l, o4l, sizeof(float) * kp, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cn4s, o4s, sizeof(float) * kp, cudaMemcpyDeviceToHost));
    return les_internal_ok();
}

les_status les_building_masks(int ip, int jp, int kp, const float *zbm, const float *z2, const float *dzn,
                              float *amask1, float *bmask1, float *cmask1, float *dmask1) {
    LES_RANGE("les_building_masks");
    if (!zbm || !z2 || !dzn || !amask1 || !bmask1 || !cmask1 || !dmask1)
        return les_internal_fail(LES_ERR_BAD_ARG, "NULL array");
    if (ip < 1 || jp < 1 || kp < 1) return les_internal_fail(LES_ERR_DIMS, "bad extents");
    const size_t nz = (size_t)(ip + 3) * (jp + 3);
    const size_t na = (size_t)(ip + 2) * (jp + 2) * (kp + 2);
    const size_t nb = (size_t)(ip + 3) * (jp + 2) * (kp + 2);
    const size_t nc = (size_t)(ip + 2) * (jp + 3) * (kp + 2);
    DevBuf d;
    CKS(cudaMalloc(&d.p, sizeof(float) * (nz + (kp + 2) + (kp + 4) + 2 * na + nb + nc)));
    float *dz = (float *)d.p, *dz2 = dz + nz, *ddzn = dz2 + kp + 2, *da = ddzn + kp + 4, *dd = da + na, *db = dd + na,
          *dc = db + nb;
    CKS(cudaMemcpy(dz, zbm, sizeof(float) * nz, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dz2, z2, sizeof(float) * (kp + 2), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(ddzn, dzn, sizeof(float) * (kp + 4), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(da, amask1, sizeof(float) * na, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dd, dmask1, sizeof(float) * na, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(db, bmask1, sizeof(float) * nb, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dc, cmask1, sizeof(float) * nc, cudaMemcpyHostToDevice));
    const size_t n = (size_t)ip * jp * kp;
    k_masks<<<(int)std::min<size_t>((n + 255) / 256, 148 * 32), 256>>>(ip, jp, kp, dz, dz2, ddzn, da, db, dc, dd);
    CKS(cudaGetLastError());
    CKS(cudaMemcpy(amask1, da, sizeof(float) * na, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(dmask1, dd, sizeof(float) * na, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(bmask1, db, sizeof(float) * nb, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(cmask1, dc, sizeof(float) * nc, cudaMemcpyDeviceToHost));
    return les_internal_ok();
}

size_t les_halo_buffer_floats(unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim, int inner) {
    if (hw == 0 || jm < 2 * hw || (inner && im < 2 * hw)) return 0;
    return halo_dims(im, jm, km, hw, vdim, inner).vsz * vdim;
}
les_status les_halo_pack(const float *a, float *b, unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim,
                         int device, void *stream) {
    LES_RANGE("les_halo_pack");
    return halo_common(a, b, im, jm, km, hw, vdim, device, stream, 0, 0);
}
les_status les_halo_unpack(float *a, const float *b, unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim,
                           int device, void *stream) {
    LES_RANGE("les_halo_unpack");
    return halo_common(b, a, im, jm, km, hw, vdim, device, stream, 0, 1);
}
// One entry per component width, named after the reference's kernels
// exchange_{1,2,4,16}_halo_read/_write (halo_exchange.cl, _correct.cl).
#define LES_HALO_WIDTH(V)                                                                                        \
    les_status les_halo_pack_##V(const float *a, float *b, unsigned im, unsigned jm, unsigned km, unsigned hw,     \
                                 int device, void *stream) {                                                     \
        return halo_common(a, b, im, jm, km, hw, V, device, stream, 0, 0);                                        \
    }                                                                                                            \
    les_status les_halo_unpack_##V(float *a, const float *b, unsigned im, unsigned jm, unsigned km, unsigned hw,   \
                                   int device, void *stream) {                                                   \
        return halo_common(b, a, im, jm, km, hw, V, device, stream, 0, 1);                                        \
    }                                                                                                            \
    les_status les_halo_pack_inner_##V(const float *a, float *b, unsigned im, unsigned jm, unsigned km,            \
                                       unsigned hw, int device, void *stream) {                                  \
        return halo_common(a, b, im, jm, km, hw, V, device, stream, 1, 0);                                        \
    }                                                                                                            \
    les_status les_halo_unpack_inner_##V(float *a, const float *b, unsigned im, unsigned jm, unsigned km,          \
                                         unsigned hw, int device, void *stream) {                                \
        return halo_common(b, a, im, jm, km, hw, V, device, stream, 1, 1);                                        \
    }
LES_HALO_WIDTH(1)
LES_HALO_WIDTH(2)
LES_HALO_WIDTH(4)
LES_HALO_WIDTH(16)
#undef LES_HALO_WIDTH

les_status les_halo_pack_inner(const float *a, float *b, unsigned im, unsigned jm, unsigned km, unsigned hw,
                               unsigned vdim, int device, void *stream) {
    LES_RANGE("les_halo_pack_inner");
    return halo_common(a, b, im, jm, km, hw, vdim, device, stream, 1, 0);
}
les_status les_halo_unpack_inner(float *a, const float *b, unsigned im, unsigned jm, unsigned km, unsigned hw,
                                 unsigned vdim, int device, void *stream) {
    LES_RANGE("les_halo_unpack_inner");
    return halo_common(b, a, im, jm, km, hw, vdim, device, stream, 1, 1);
}

// ---------------------------------------------------------------- synthetic
// (les_synth_gen.h, shared with the CPU oracle)
void les_synth_default(les_synth_cfg *c, int ip, int jp, int kp, uint64_t seed) {
    les_synth_gen::defaults(c, ip, jp, kp, seed);
}

les_status les_synth_grid(const les_synth_cfg *c, float *dx1, float *dxl, float *dy1, float *dyl, float *z2,
                          float *dzn, float *dzs, float *dxs, float *dys) {
    LES_RANGE("les_synth_grid");
    if (!c || !dx1 || !dy1 || !dzn) return les_internal_fail(LES_ERR_BAD_ARG, "NULL argument");
    les_synth_gen::base_grid(c, dx1, dy1, dzn);
    return les_grid_metrics(c->ip, c->jp, c->kp, dx1, dxl, dy1, dyl, z2, dzn, dzs, dxs, dys);
}

float les_synth_terrain(const les_synth_cfg *c, float *zbm) { return les_synth_gen::terrain(c, zbm); }

les_status les_synth_inflow(const les_synth_cfg *c, const float *z2, const float *dzn, float *wp) {
    LES_RANGE("les_synth_inflow");
    if (!c || !z2 || !dzn || !wp) return les_internal_fail(LES_ERR_BAD_ARG, "NULL argument");
    les_synth_gen::inflow(c, z2, dzn, wp);
    return les_internal_ok();
}

}  // extern "C"
