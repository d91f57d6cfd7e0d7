// les_noalloc.cu -- press.f95:49-81 (bondfg, rhs, rhsav and its
// subtraction) on arrays the caller already holds on the device, allocating
// no device memory.
//
// It serves hosts that cannot allocate in their time loop: a host whose
// memory pool already holds the free device memory (cudaMalloc fails there)
// or one that overlaps work on other streams (cudaFree synchronises the
// device).  The exact global sums need per-block partials.  They live in one
// file-scope static __device__ array (kScratchBytes, held by every GPU that
// loads the library until the process exits); the host looks up its
// address once per device with cudaGetSymbolAddress and never calls
// cudaMalloc, cudaFree or a library routine that allocates.  Layout of the
// scratch:
//   bytes [0, 4)      ticket: blocks of the current call that have finished.
//                     Must be zero when a call starts; static storage is
//                     zero at module load and the last block of every call
//                     sets it back to zero.
//   bytes [4, 8)      rhsav of the current call (written by the last block).
//   bytes [256, ...)  two FixParts per block (sum of dx1*dy1*dzn*rhs, sum
//                     of dx1*dy1*dzn); written before they are read, so
//                     their contents between calls do not matter.
// One scratch serves all calls on a device: calls that overlap in time on
// the same device (two streams, two host threads) race on it.  The looked-up
// address is kept per device for the life of the process, which assumes one
// primary context per device: a cudaDeviceReset unloads the module and
// leaves the kept address stale (documented at the declaration).
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "les_abi.h"
#include "les_dev.cuh"

les_status les_internal_fail(les_status s, const char *msg);
les_status les_internal_ok();

namespace {

constexpr size_t kScratchBytes = 256 * 1024;
constexpr size_t kScratchHead = 256;
constexpr int kNaBX = 32, kNaBY = 8, kNaNT = kNaBX * kNaBY;
constexpr int kNaMaxBlocks = (int)((kScratchBytes - kScratchHead) / (2 * sizeof(les::FixPart)));
constexpr int kNaMaxDev = 64;

}  // namespace

static __device__ __align__(256) unsigned char les_press_rhs_scratch[kScratchBytes];

namespace {

using les::FixPart;
using les::i128;

// Fortran layouts of press.f95:11-35 (ip = im, jp = jm, kp = km).
struct PressRhsDims {
    int im, jm, km;
    __device__ long long fgh(int i, int j, int k) const {  // (0:ip, 0:jp, 0:kp)
        return i + (long long)(im + 1) * (j + (long long)(jm + 1) * k);
    }
    __device__ long long rhs(int i, int j, int k) const {  // (0:ip+1, 0:jp+1, 0:kp+1)
        return i + (long long)(im + 2) * (j + (long long)(jm + 2) * k);
    }
    __device__ long long uv(int i, int j, int k) const {  // (0:ip+1, -1:jp+1, 0:kp+1)
        return i + (long long)(im + 2) * ((j + 1) + (long long)(jm + 3) * k);
    }
    __device__ long long w(int i, int j, int k) const {  // (0:ip+1, -1:jp+1, -1:kp+1)
        return i + (long long)(im + 2) * ((j + 1) + (long long)(jm + 3) * (k + 1));
    }
};

__device__ __forceinline__ FixPart load_part_cg(const FixPart *p) {
    FixPart q;
    q.lo = __ldcg(&p->lo);
    q.hi = __ldcg(&p->hi);
    q.bad = __ldcg(&p->bad);
    q.pad = 0;
    return q;
}

// bondFG.f95:15-31 and press.f95:51-62 for the columns of a 32 x 8 tile and
// a chunk of k, then the partial sums of press.f95:65-74; the last block to
// finish adds all partials and forms rhsav (press.f95:75).  Same expression
// order as the context path's k_rhs.
__global__ void __launch_bounds__(kNaNT)
    k_press_rhs_na(PressRhsDims d, float *__restrict__ rhs, const float *__restrict__ u,
                   const float *__restrict__ v, const float *__restrict__ w, float *__restrict__ f,
                   float *__restrict__ g, float *__restrict__ h, const float *__restrict__ dx1p,
                   const float *__restrict__ dy1, const float *__restrict__ dznp, float dt, int kchunk,
                   unsigned char *scratch) {
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch);
    float *rhsav_slot = reinterpret_cast<float *>(scratch + 4);
    FixPart *part = reinterpret_cast<FixPart *>(scratch + kScratchHead);
    const float *dx1 = dx1p + 1, *dzn = dznp + 1;  // dx1(-1:ip+1), dzn(-1:kp+2)
    const int i = 1 + blockIdx.x * kNaBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kNaBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(d.km, k0 + kchunk - 1);
    i128 num = 0, area = 0;
    int bad_num = 0, bad_area = 0;
    if (i <= d.im && j <= d.jm) {
        for (int k = k0; k <= k1; ++k) {
            const long long c = d.fgh(i, j, k);
            const float fc = f[c], gc = g[c];
            float hc = h[c];
            // bondfg: f(0,j,k)=f(1,j,k); g(i,0,k)=g(i,jm,k); h(i,j,0)=h(i,j,km)=0
            if (i == 1) f[d.fgh(0, j, k)] = fc;
            if (j == d.jm) g[d.fgh(i, 0, k)] = gc;
            if (k == d.km) {
                h[c] = 0.0f;
                hc = 0.0f;
            }
            if (k == 1) h[d.fgh(i, j, 0)] = 0.0f;
            const float fm = (i == 1) ? fc : f[d.fgh(i - 1, j, k)];
            const float gm = (j == 1) ? g[d.fgh(i, d.jm, k)] : g[d.fgh(i, j - 1, k)];
            const float hm = (k == 1) ? 0.0f : h[d.fgh(i, j, k - 1)];
            float r = (-u[d.uv(i - 1, j, k)] + u[d.uv(i, j, k)]) / dx1[i] +
                      (-v[d.uv(i, j - 1, k)] + v[d.uv(i, j, k)]) / dy1[j] +
                      (-w[d.w(i, j, k - 1)] + w[d.w(i, j, k)]) / dzn[k];
            r = (fc - fm) / dx1[i] + (gc - gm) / dy1[j] + (hc - hm) / dzn[k] + r / dt;
            rhs[d.rhs(i, j, k)] = r;
            num += les::fix_term(dx1[i] * dy1[j] * dzn[k] * r, bad_num);
            area += les::fix_term(dx1[i] * dy1[j] * dzn[k], bad_area);
        }
    }
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    les::block_fix_sum<kNaNT>(num, bad_num, &part[2 * b]);
    __syncthreads();  // block_fix_sum's shared words are reused below
    les::block_fix_sum<kNaNT>(area, bad_area, &part[2 * b + 1]);
    __shared__ int s_last;
    const int t = threadIdx.x + kNaBX * threadIdx.y;
    if (t == 0) {
        __threadfence();  // this block's partials before its ticket
        s_last = (atomicAdd(ticket, 1u) == (unsigned int)nblocks - 1u);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    i128 tn = 0, ta = 0;
    int bn = 0, ba = 0;
    for (int q = t; q < nblocks; q += kNaNT) {
        const FixPart pn = load_part_cg(&part[2 * q]), pa = load_part_cg(&part[2 * q + 1]);
        tn += les::fix_from_part(pn);
        bn |= pn.bad;
        ta += les::fix_from_part(pa);
        ba |= pa.bad;
    }
    __shared__ FixPart s_tot[2];
    __syncthreads();
    les::block_fix_sum<kNaNT>(tn, bn, &s_tot[0]);
    __syncthreads();
    les::block_fix_sum<kNaNT>(ta, ba, &s_tot[1]);
    if (t == 0) {
        const double sn = les::fix_finish(les::fix_from_part(s_tot[0]), s_tot[0].bad);
        const double sa = les::fix_finish(les::fix_from_part(s_tot[1]), s_tot[1].bad);
        *rhsav_slot = (float)(sn / sa);
        *ticket = 0u;  // ready for the next call
    }
}

// press.f95:76-81: rhs(i,j,k) = rhs(i,j,k) - rhsav on the interior.
__global__ void __launch_bounds__(kNaNT) k_press_rhs_sub_na(PressRhsDims d, float *__restrict__ rhs, int kchunk,
                                                            const unsigned char *scratch, float *rhsav_out) {
    const float rhsav = *reinterpret_cast<const float *>(scratch + 4);
    const int i = 1 + blockIdx.x * kNaBX + threadIdx.x;
    const int j = 1 + blockIdx.y * kNaBY + threadIdx.y;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(d.km, k0 + kchunk - 1);
    if (rhsav_out && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) *rhsav_out = rhsav;
    if (i > d.im || j > d.jm) return;
    for (int k = k0; k <= k1; ++k) {
        const long long c = d.rhs(i, j, k);
        rhs[c] = rhs[c] - rhsav;
    }
}

std::mutex g_na_mu;
unsigned char *g_na_addr[kNaMaxDev];

les_status na_fail(les_status s, const char *fmt, long long a = 0, long long b = 0) {
    char buf[256];
    std::snprintf(buf, sizeof buf, fmt, a, b);
    return les_internal_fail(s, buf);
}

}  // namespace

extern "C" les_status les_press_rhs_noalloc(int km, int jm, int im, float *rhs, const float *u, const float *dx1,
                                            const float *v, const float *dy1, const float *w, const float *dzn,
                                            float *f, float *g, float *h, float dt, float *rhsav, void *stream) {
    if (!rhs || !u || !dx1 || !v || !dy1 || !w || !dzn || !f || !g || !h)
        return les_internal_fail(LES_ERR_BAD_ARG, "les_press_rhs_noalloc: NULL array");
    if (im < 1 || jm < 1 || km < 1) return les_internal_fail(LES_ERR_DIMS, "les_press_rhs_noalloc: im, jm, km < 1");
    const long long gx = (im + kNaBX - 1) / kNaBX, gy = (jm + kNaBY - 1) / kNaBY;
    if (gx * gy > kNaMaxBlocks)
        return na_fail(LES_ERR_DIMS,
                       "les_press_rhs_noalloc: %lld tiles of 32 x 8 columns exceed the %lld the static scratch "
                       "holds (ceil(im/32) * ceil(jm/8) must be <= that)",
                       gx * gy, (long long)kNaMaxBlocks);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return na_fail(LES_ERR_CUDA, "les_press_rhs_noalloc: no CUDA device");
    }
    if (dev < 0 || dev >= kNaMaxDev) return na_fail(LES_ERR_CUDA, "les_press_rhs_noalloc: device %lld", dev);
    unsigned char *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_addr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, les_press_rhs_scratch);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return na_fail(LES_ERR_CUDA, "les_press_rhs_noalloc: scratch address lookup failed");
            }
            g_na_addr[dev] = static_cast<unsigned char *>(p);
        }
        scratch = g_na_addr[dev];
    }
    // >= 4 blocks per SM when the (i,j) tiles alone are fewer, within the scratch
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long nk = (4LL * nsm + gx * gy - 1) / (gx * gy);
    nk = nk < 1 ? 1 : (nk > km ? km : nk);
    if (gx * gy * nk > kNaMaxBlocks) nk = kNaMaxBlocks / (gx * gy);
    const int kchunk = (int)((km + nk - 1) / nk);
    nk = (km + kchunk - 1) / kchunk;
    const PressRhsDims d{im, jm, km};
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)nk), block(kNaBX, kNaBY);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_press_rhs_na<<<grid, block, 0, st>>>(d, rhs, u, v, w, f, g, h, dx1, dy1, dzn, dt, kchunk, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return les_internal_fail(LES_ERR_CUDA, cudaGetErrorString(e));
    k_press_rhs_sub_na<<<grid, block, 0, st>>>(d, rhs, kchunk, scratch, rhsav);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return les_internal_fail(LES_ERR_CUDA, cudaGetErrorString(e));
    return les_internal_ok();
}
