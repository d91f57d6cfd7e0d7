// les_lib.cu -- host side of liblesb200.so: contexts, the host boundary,
// the graph-captured time step and the setup routines (les_abi.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "les_abi.h"
#include "les_adjoint.cuh"
#include "les_adjstep.cuh"
#include "les_halo.cuh"
#include "les_mom.cuh"
#include "les_press.cuh"
#include "les_routines.cuh"
#include "les_sor_tb.cuh"
#include "les_sor1.cuh"
#include "les_sor1p.cuh"
#include "les_stats.cuh"
#include "les_refine.cuh"
#include "les_spectral.cuh"
#include "les_fft.cuh"
#include "les_nvtx.h"
#include "les_step.cuh"
#include "les_dd.cuh"

using namespace les;

namespace {

thread_local std::string g_err;

les_status fail(les_status s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}
les_status ok() {
    g_err.clear();
    return LES_OK;
}

}  // namespace

les_status les_internal_fail(les_status s, const char *msg) { return fail(s, "%s", msg); }
les_status les_internal_ok() { return ok(); }

namespace {

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(LES_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define CKL()                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) return fail(LES_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e_)); \
    } while (0)

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// Fortran bounds of each state field (main_ocl.f95:41-167).
struct FBounds {
    int li, ui, lj, uj, lk, uk;
    int ni() const { return ui - li + 1; }
    int nj() const { return uj - lj + 1; }
    int nk() const { return uk - lk + 1; }
    size_t n() const { return (size_t)ni() * nj() * nk(); }
};
FBounds field_bounds(int f, int ip, int jp, int kp) {
    switch (f) {
        case LES_F_U:
        case LES_F_V: return {0, ip + 1, -1, jp + 1, 0, kp + 1};
        case LES_F_W: return {0, ip + 1, -1, jp + 1, -1, kp + 1};
        case LES_F_P: return {0, ip + 2, 0, jp + 2, 0, kp + 1};
        case LES_F_USUM:
        case LES_F_VSUM:
        case LES_F_WSUM:
        case LES_F_F:
        case LES_F_G:
        case LES_F_H: return {0, ip, 0, jp, 0, kp};
        case LES_F_FOLD:
        case LES_F_GOLD:
        case LES_F_HOLD: return {1, ip, 1, jp, 1, kp};
        case LES_F_RHS: return {0, ip + 1, 0, jp + 1, 0, kp + 1};
        case LES_F_SM: return {-1, ip + 1, -1, jp + 1, 0, kp + 1};
        case LES_F_AMASK:
        case LES_F_DMASK: return {0, ip + 1, 0, jp + 1, 0, kp + 1};
        case LES_F_BMASK: return {-1, ip + 1, 0, jp + 1, 0, kp + 1};
        case LES_F_CMASK: return {0, ip + 1, -1, jp + 1, 0, kp + 1};
    }
    return {0, 0, 0, 0, 0, 0};
}

// Offsets of the 1-D tables inside one device buffer (each with slack).
struct TableLayout {
    size_t dx1, dy1, dzn, dzs, dxs, dys, cn2l, cn2s, cn3l, cn3s, cn4l, cn4s, cnA, cnB, cnC, smc, wind;
    size_t rdx1, rsx, rdy1, rsy, cn1k, rdzn, rdzs, rdzn2, total;
};
TableLayout table_layout(int ip, int jp, int kp) {
    TableLayout t;
    size_t o = 0;
    auto take = [&](size_t n) {
        size_t r = o;
        o += (n + 31) / 32 * 32;
        return r;
    };
    t.dx1 = take(ip + 4);
    t.dy1 = take(jp + 4);
    t.dzn = take(kp + 5);
    t.dzs = take(kp + 5);
    t.dxs = take(ip + 2);
    t.dys = take(jp + 2);
    t.cn2l = take(ip + 2);
    t.cn2s = take(ip + 2);
    t.cn3l = take(jp + 2);
    t.cn3s = take(jp + 2);
    t.cn4l = take(kp + 2);
    t.cn4s = take(kp + 2);
    t.cnA = take(ip + 2);
    t.cnB = take(jp + 2);
    t.cnC = take(kp + 2);
    t.smc = take(kp + 2);
    t.wind = take((size_t)jp * kp);
    t.rdx1 = take(ip + 4);
    t.rsx = take(ip + 4);
    t.rdy1 = take(jp + 4);
    t.rsy = take(jp + 4);
    t.cn1k = take(kp + 2);
    t.rdzn = take(kp + 5);
    t.rdzs = take(kp + 5);
    t.rdzn2 = take(kp + 5);
    t.total = o;
    return t;
}

}  // namespace

// Shape of a temporal-blocked SOR pass: iterations per pass, tile rows,
// k chunks.
struct TbShape {
    int T = 0, ty = 0, nch = 1;
    int rows = 1;  // region rows per warp: 2 takes k_sor1p (T = 1, ty + 4 even)
};

struct SpecState;  // spectral solve of the refined press (les_refine.inc)
void spec_release(SpecState *s);

struct les_ctx {
    les_params prm{};
    Geo geo{};
    Fields F{};
    float *d_fields = nullptr;
    size_t box_elems = 0;
    float *d_tables = nullptr;
    TableLayout tl{};
    std::vector<float> h_tables;
    Scal *d_scal = nullptr;
    FixPart *d_part = nullptr;
    int npart = 0;
    float *d_stage = nullptr;
    size_t stage_elems = 0;
    cudaStream_t stream = nullptr;
    // step graphs: index = (n==1 broadcast) + 2 * (exact per-colour SOR)
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaGraph_t graph_src[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t graph_kernels[4] = {0, 0, 0, 0};
    // per-step phase timing (les_ctx_set_timing): event record nodes in the
    // step graphs are pointed at slot `tslot` before each launch
    int tslots = 0, tslot = 0;
    std::vector<cudaEvent_t> tev;  // tslots x LES_NTEV
    std::vector<cudaGraphNode_t> tnode[4];
    std::vector<int> tnode_idx[4];
    bool capturing_timed = false;
    double area = 0.0;
    uint64_t launches = 0;
    bool uploaded = false;
    bool rhs_raw = false;  // interior of rhs holds values before the rhsav subtraction
    int red_gx = 0, red_gy = 0, red_nk = 0, red_kchunk = 0;
    int last_n = 0;
    std::vector<float *> extra;      // scratch boxes of the per-routine entries
    const float *cn1_box = nullptr;  // caller's cn1 (per-routine press only)
    // temporal-blocked SOR (les_sor_tb.cuh)
    float *d_p2 = nullptr;           // second p buffer
    TbShape tb;  // SOR pass shape chosen by the autotuner (tb.T == 0: not yet)
    bool xy_pow2 = false;  // every x/y spacing divisor a power of two (build_tables)
    bool cn1_by_k = false;           // uniform dx, dy: cn1 from a per-k table
    bool p_ghosts_ok = false;        // p's ghosts hold what boundp1/boundp2 give
    bool force_exact_sor = false;    // testing: always the per-colour path
    bool sor_fp32_test = true;       // LES_SOR_SUMS=exact clears it: every pass sums exactly
    float *d_ave = nullptr;          // aveflow statistics (les_stats.cuh), allocated on first use
    TbKCoef kq{};                    // per-plane SOR coefficients (build_tables), a pass kernel's parameter
    unsigned table_gen = 0;          // bumped whenever build_tables runs (captured graphs are dropped)
    // FP64-refined press (les_refine.cuh): corrections per step, inner sweeps, tolerance
    int ref_outer = 0, ref_inner = 0;
    double ref_tol = 0.0;
    double *d_p64 = nullptr;              // FP64 p (box)
    float *d_r32 = nullptr, *d_e0 = nullptr, *d_e1 = nullptr;  // inner rhs and correction buffers
    Scal *d_scal2 = nullptr;              // scalars of the inner sweeps
    Ref64 *d_ref = nullptr;
    double2 *d_dpart = nullptr;           // FP64 per-block partial sums
    double *d_refw = nullptr;             // left null vector weights wx, wy, wz
    SpecState *spec = nullptr;            // spectral inner solve (inner = 0)
    // reduction mode (les_ctx_set_reduction_mode): LES_RED_F_* bits take
    // rhsav, the SOR residual or pav in the reference's sequential FP32 order
    int red_mode = LES_RED_CANONICAL;
    float *d_r2 = nullptr;                // reltmp^2 per cell (box), LES_RED_F_SOR only
    float *d_drag = nullptr;              // per-column IBM force scale (les_ctx_set_drag)
    // x-decomposed domain (les_dd.inc): this context is one rank's slab
    bool dd = false;
    bool dd_passes = false;               // its SOR on one-iteration passes (else per colour)
    double dd_area = 0.0;                 // the whole domain's rhsav/pav denominator
    long long *d_dd = nullptr;            // limbs of a global sum (kDDLimbs)
    cudaEvent_t dd_ev = nullptr;          // orders les_dd_local_sum against this context's stream
};

// Buffers of an SOR pass other than the context's p / second p / rhs / scalars.
struct SorBufs {
    float *pb0, *pb1;
    const float *rhs;
    Scal *sc;
};

namespace {

float *field_ptr(les_ctx *c, int f) { return c->d_fields + (size_t)f * c->box_elems; }
les_status launch_sor_tb(les_ctx *c, const TbShape &sh, int niter, int mode, float pjuge, int itmax,
                         bool tuning = false, const SorBufs *bufs = nullptr);

// The SOR of the next step runs one colour sweep at a time (press.f95's own
// sequence with materialised ghosts) instead of the temporal-blocked passes:
// on request, for odd jp below the shortest one-iteration pass region
// (odd jp takes one-iteration passes only, whose region must not hold a row
// twice), for a just-uploaded p whose ghosts are not boundary-consistent,
// for km >= kTbKMax, and for reference-order residual sums.
bool sor_per_colour(const les_ctx *c) {
    return c->force_exact_sor || ((c->prm.jp % 2) != 0 && c->prm.jp < tb_rh(1, 4)) || !c->p_ghosts_ok ||
           c->prm.kp >= kTbKMax || (c->red_mode & LES_RED_F_SOR);
}

void drop_step_graphs(les_ctx *c) {
    for (int gi = 0; gi < 4; ++gi) {
        if (c->graph[gi]) cudaGraphExecDestroy(c->graph[gi]);
        if (c->graph_src[gi]) cudaGraphDestroy(c->graph_src[gi]);
        c->graph[gi] = nullptr;
        c->graph_src[gi] = nullptr;
        c->tnode[gi].clear();
        c->tnode_idx[gi].clear();
    }
}
les_status enqueue_refine(les_ctx *c);
bool tb_fast_ok(const les_ctx *c, const TbShape &sh);

// Host copies of the 1-D tables -> device; builds cnA/B/C, smc, wind.
// Tables not given stay zero (the per-routine entries pass only theirs).
// y = RN(1/b) for kdiv, or 0 when b is outside [2^-30, 2^30] (or not
// finite), which makes kdiv divide.
float kdiv_recip(float b) {
    const float a = std::fabs(b);
    return (a >= 0x1p-30f && a <= 0x1p30f) ? 1.0f / b : 0.0f;
}

les_status build_tables(les_ctx *c, const les_host_fields *hf, bool require_inflow) {
    const int ip = c->prm.ip, jp = c->prm.jp, kp = c->prm.kp;
    const TableLayout &t = c->tl;
    std::vector<float> &h = c->h_tables;
    h.assign(t.total, 0.0f);
    auto cp = [&](size_t off, const float *src, size_t n) {
        if (src) std::memcpy(&h[off], src, n * sizeof(float));
    };
    cp(t.dx1, hf->dx1, ip + 3);  // -1..ip+1
    cp(t.dy1, hf->dy1, jp + 2);  // 0..jp+1
    cp(t.dzn, hf->dzn, kp + 4);  // -1..kp+2
    cp(t.dzs, hf->dzs, kp + 4);
    cp(t.dxs, hf->dxs, ip + 1);  // 0..ip
    cp(t.dys, hf->dys, jp + 1);
    cp(t.cn2l, hf->cn2l, ip);  // 1..ip
    cp(t.cn2s, hf->cn2s, ip);
    cp(t.cn3l, hf->cn3l, jp);
    cp(t.cn3s, hf->cn3s, jp);
    cp(t.cn4l, hf->cn4l, kp);
    cp(t.cn4s, hf->cn4s, kp);
    auto dx1 = [&](int i) { return h[t.dx1 + i + 1]; };
    auto dy1 = [&](int j) { return h[t.dy1 + j]; };
    auto dzn = [&](int k) { return h[t.dzn + k + 1]; };
    auto dzs = [&](int k) { return h[t.dzs + k + 1]; };
    auto dxs = [&](int i) { return h[t.dxs + i]; };
    auto dys = [&](int j) { return h[t.dys + j]; };
    // init.f95:87-93 separable parts of cn1
    for (int i = 1; i <= ip; ++i) h[t.cnA + i - 1] = 2.0f / (dxs(i - 1) * dxs(i));
    for (int j = 1; j <= jp; ++j) h[t.cnB + j - 1] = 2.0f / (dys(j - 1) * dys(j));
    for (int k = 1; k <= kp; ++k) h[t.cnC + k - 1] = 2.0f / (dzs(k - 1) * dzs(k));
    // les.f95:125-129, 146-148
    for (int k = 1; k <= kp; ++k) {
        const float delx1 = powf(dx1(0) * dy1(0) * dzn(k), 1.0f / 3.0f);
        const float cd = c->prm.cs0 * delx1;
        h[t.smc + k - 1] = cd * cd;
    }
    // inflow table: bondv1.f95:26-45 power law or the external profile
    if (c->prm.inflow_mode == LES_INFLOW_EXTERNAL) {
        if (!hf->wind_profile && require_inflow) return fail(LES_ERR_BAD_ARG, "external inflow needs wind_profile");
        if (hf->wind_profile) std::memcpy(&h[t.wind], hf->wind_profile, sizeof(float) * (size_t)jp * kp);
    } else if (hf->z2 || require_inflow) {
        if (!hf->z2) return fail(LES_ERR_BAD_ARG, "power-law inflow needs z2");
        std::vector<float> col(kp + 1);
        for (int k = 1; k <= kp; ++k) {
            if (k <= 78) {
                col[k] = 5.0f * powf((hf->z2[k - 1] + 0.5f * dzn(k)) / 600.0f, 0.2f);
            } else {
                col[k] = col[77];
            }
        }
        for (int k = 1; k <= kp; ++k)
            for (int j = 1; j <= jp; ++j) h[t.wind + (j - 1) + (size_t)jp * (k - 1)] = col[k];
    }
    // cn1 depends on k only when cnA and cnB are constant (uniform dx, dy):
    // cn1k(k) = 1/((cnA+cnB)+cnC(k)) is then bit-identical to init.f95:87-93
    {
        bool uni = true;
        for (int i = 2; i <= ip && uni; ++i) uni = std::memcmp(&h[t.cnA], &h[t.cnA + i - 1], 4) == 0;
        for (int j = 2; j <= jp && uni; ++j) uni = std::memcmp(&h[t.cnB], &h[t.cnB + j - 1], 4) == 0;
        c->cn1_by_k = uni && hf->dxs && hf->dys && hf->dzs;
        for (int k = 1; k <= kp; ++k) h[t.cn1k + k] = 1.0f / (h[t.cnA] + h[t.cnB] + h[t.cnC + k - 1]);
    }
    c->kq = TbKCoef{};
    for (int k = 1; k <= kp && k < kTbKMax; ++k) {
        c->kq.c4l[k] = h[t.cn4l + k - 1];
        c->kq.c4s[k] = h[t.cn4s + k - 1];
        c->kq.cnk[k] = c->cn1_by_k ? h[t.cn1k + k] : 0.0f;
    }
    // graphs captured before hold the old tables' kernel choices and
    // parameters: capture again at the next step
    drop_step_graphs(c);
    ++c->table_gen;
    // exact reciprocals of power-of-two x/y divisors (0 otherwise)
    auto recip = [](float d) -> float {
        int e = 0;
        const float m = std::frexp(d, &e);
        if (!(d > 0.0f) || m != 0.5f || e < -120 || e > 120) return 0.0f;
        return std::ldexp(1.0f, 1 - e);  // d = 2^(e-1)
    };
    for (int i = -1; i <= ip + 1; ++i) h[t.rdx1 + i + 1] = recip(dx1(i));
    for (int i = -1; i <= ip; ++i) h[t.rsx + i + 1] = recip(dx1(i) + dx1(i + 1));
    for (int j = 0; j <= jp + 1; ++j) h[t.rdy1 + j] = recip(dy1(j));
    for (int j = 0; j <= jp; ++j) h[t.rsy + j] = recip(dy1(j) + dy1(j + 1));
    // reciprocals of the k divisors for kdiv
    for (int k = -1; k <= kp + 2; ++k) {
        h[t.rdzn + k + 1] = kdiv_recip(dzn(k));
        h[t.rdzs + k + 1] = kdiv_recip(dzs(k));
        if (k <= kp + 1) h[t.rdzn2 + k + 1] = kdiv_recip(dzn(k) + dzn(k + 1));
    }
    // every x/y divisor of the face and cell formulas a power of two: the tile
    // engine multiplies by the reciprocal without testing it
    c->xy_pow2 = true;
    for (int i = -1; i <= ip + 1; ++i) c->xy_pow2 = c->xy_pow2 && h[t.rdx1 + i + 1] != 0.0f;
    for (int i = -1; i <= ip; ++i) c->xy_pow2 = c->xy_pow2 && h[t.rsx + i + 1] != 0.0f;
    for (int j = 0; j <= jp + 1; ++j) c->xy_pow2 = c->xy_pow2 && h[t.rdy1 + j] != 0.0f;
    for (int j = 0; j <= jp; ++j) c->xy_pow2 = c->xy_pow2 && h[t.rsy + j] != 0.0f;
    // grid-only denominator of rhsav and pav (press.f95:134, 192)
    i128 acc = 0;
    int bad = 0;
    for (int k = 1; k <= kp; ++k)
        for (int j = 1; j <= jp; ++j)
            for (int i = 1; i <= ip; ++i) acc += fix_term(dx1(i) * dy1(j) * dzn(k), bad);
    c->area = fix_finish(acc, bad);
    CK(cudaMemcpyAsync(c->d_tables, h.data(), sizeof(float) * t.total, cudaMemcpyHostToDevice, c->stream));
    return ok();
}

// Phase boundaries recorded by the timing events (les_ctx_phase_times).
enum { EV_START = 0, EV_BONDV1, EV_VELFG, EV_VISC, EV_RHS, EV_SOR1_START, EV_SOR1_END, EV_SOR_END, EV_PAV, LES_NTEV };

les_status mark(les_ctx *c, int which) {
    if (!c->capturing_timed) return LES_OK;
    CK(cudaEventRecordWithFlags(c->tev[which], c->stream, cudaEventRecordExternal));
    return LES_OK;
}
#define MARK(c, w)                                     \
    do {                                               \
        les_status ms_ = mark((c), (w));               \
        if (ms_ != LES_OK) return ms_;                 \
    } while (0)

// Kernel launch helpers; each counts one launch.
#define LAUNCH(c, kern, grid, block, ...)                          \
    do {                                                           \
        kern<<<(grid), (block), 0, (c)->stream>>>(__VA_ARGS__);    \
        CKL();                                                     \
        ++(c)->launches;                                           \
    } while (0)
#define LAUNCH_SMEM(c, kern, grid, block, smem, ...)                  \
    do {                                                              \
        kern<<<(grid), (block), (smem), (c)->stream>>>(__VA_ARGS__);  \
        CKL();                                                        \
        ++(c)->launches;                                              \
    } while (0)

dim3 cells_grid(const Geo &g, int i0) {  // i from i0, 32 x 4 blocks, z = k
    return dim3(cdiv(g.im - i0 + 1, 32), cdiv(g.jm, 4), g.km);
}

les_status enqueue_bondv1(les_ctx *c, int n, bool velnw) {
    const Geo &g = c->geo;
    if (velnw)
        LAUNCH(c, k_velnw_inflow<true>, cells_grid(g, 1), dim3(32, 4), g, c->F, n, c->prm.ical);
    else
        LAUNCH(c, k_velnw_inflow<false>, cells_grid(g, 1), dim3(32, 4), g, c->F, n, c->prm.ical);
    LAUNCH(c, k_uout_reduce, dim3(cdiv((long long)g.jm * g.km, 256 * 8)), dim3(256), g, c->F.u, c->d_scal);
    LAUNCH(c, k_outflow, dim3(cdiv((long long)g.jm * g.km, 256)), dim3(256), g, c->F, c->d_scal);
    const long long ng = 2LL * g.km * (g.im + 2) + 2LL * (g.jm + 2) * (g.im + 2) + 2LL * (g.jm + 3) * (g.im + 2);
    LAUNCH(c, k_uvw_ghosts, dim3(cdiv(ng, 256)), dim3(256), g, c->F);
    return LES_OK;
}

les_status enqueue_velfg_les(les_ctx *c, bool adam) {
    const Geo &g = c->geo;
    const dim3 mg(cdiv(g.im, kMX), cdiv(g.jm, kMY));
    const bool band = g.jm >= kBH;  // the staged band must not wrap onto itself
    const bool p2 = band && c->xy_pow2;
    if (p2)
        LAUNCH_SMEM(c, (k_mom1<true, true>), mg, dim3(kMNT), mom_smem(false), g, c->F);
    else if (band)
        LAUNCH_SMEM(c, (k_mom1<true, false>), mg, dim3(kMNT), mom_smem(false), g, c->F);
    else
        LAUNCH_SMEM(c, (k_mom1<false, false>), mg, dim3(kMNT), mom_smem(false), g, c->F);
    MARK(c, EV_VELFG);
    const long long nb = 2LL * (g.jm + 3) * (g.km + 2) + 2LL * g.im * (g.km + 2) + 2LL * g.im * (g.jm + 1);
    LAUNCH(c, k_boundsm, dim3(cdiv(nb, 256)), dim3(256), g, c->F.sm);
    const size_t sm2 = mom_smem(true);
#define M2(A, B, P) LAUNCH_SMEM(c, (k_mom2<A, B, P>), mg, dim3(kMNT), sm2, g, c->F)
    if (adam) {
        if (p2)
            M2(true, true, true);
        else if (band)
            M2(true, true, false);
        else
            M2(true, false, false);
    } else {
        if (p2)
            M2(false, true, true);
        else if (band)
            M2(false, true, false);
        else
            M2(false, false, false);
    }
#undef M2
    MARK(c, EV_VISC);
    return LES_OK;
}

les_status enqueue_boundp(les_ctx *c, bool check) {
    const Geo &g = c->geo;
    const long long n1 = 2LL * (g.jm + 2) * (g.km + 2) + 2LL * g.im * (g.km + 2);
    const long long n2 = 2LL * (g.im + 2) * (g.jm + 2);
    if (check) {
        LAUNCH(c, k_boundp1<true>, dim3(cdiv(n1, 256)), dim3(256), g, c->F.p, c->d_scal);
    } else {
        LAUNCH(c, k_boundp1<false>, dim3(cdiv(n1, 256)), dim3(256), g, c->F.p, c->d_scal);
        LAUNCH(c, k_boundp2<false>, dim3(cdiv(n2, 256)), dim3(256), g, c->F.p, c->d_scal);
    }
    return LES_OK;
}

// press.f95:49-146.  exact=true: per-colour sweeps with materialised
// boundp1/boundp2 ghosts (any jm, any ghost state); otherwise the
// temporal-blocked sweeps of les_sor_tb.cuh (even jm, consistent ghosts).
les_status enqueue_press(les_ctx *c, bool exact) {
    const Geo &g = c->geo;
    const dim3 rg(c->red_gx, c->red_gy, c->red_nk), rb(kRedBX, kRedBY);
    const int np = c->red_gx * c->red_gy * c->red_nk;
    const long long n1 = 2LL * (g.jm + 2) * (g.km + 2) + 2LL * g.im * (g.km + 2);
    const long long n2 = 2LL * (g.im + 2) * (g.jm + 2);
    LAUNCH(c, k_rhs, rg, rb, g, c->F, c->red_kchunk, c->d_part);
    if (c->red_mode & LES_RED_F_RHSAV)
        LAUNCH(c, k_seq_sum<0>, dim3(1), dim3(kSeqNT), g, c->F.rhs, nullptr, 0.0f, c->d_scal);
    else
        LAUNCH(c, k_final_rhsav, dim3(1), dim3(1024), c->d_part, np, c->area, c->d_scal);
    if (c->ref_outer > 0) LAUNCH(c, k_ref_rhsav, dim3(1), dim3(1024), c->d_part, np, c->area, c->d_ref);
    MARK(c, EV_RHS);
    if (exact) {
        for (int l = 0; l < c->prm.nmaxp; ++l) {
            for (int nrd = 0; nrd <= 1; ++nrd) {
                if (l == 0 && nrd == 0) MARK(c, EV_SOR1_START);
                if (c->cn1_box)
                    LAUNCH(c, k_sor_colour<true>, rg, rb, g, c->F.p, c->F.rhs, c->cn1_box, nrd, c->red_kchunk,
                           c->d_part + nrd * np, c->d_scal, c->d_r2);
                else
                    LAUNCH(c, k_sor_colour<false>, rg, rb, g, c->F.p, c->F.rhs, nullptr, nrd, c->red_kchunk,
                           c->d_part + nrd * np, c->d_scal, c->d_r2);
                if (l == 0 && nrd == 0) MARK(c, EV_SOR1_END);
                LAUNCH(c, k_boundp1<true>, dim3(cdiv(n1, 256)), dim3(256), g, c->F.p, c->d_scal);
            }
            LAUNCH(c, k_boundp2<true>, dim3(cdiv(n2, 256)), dim3(256), g, c->F.p, c->d_scal);
            if (c->red_mode & LES_RED_F_SOR)
                LAUNCH(c, k_seq_sum<1>, dim3(1), dim3(kSeqNT), g, c->d_r2, nullptr, c->prm.pjuge, c->d_scal);
            else
                LAUNCH(c, k_final_sor, dim3(1), dim3(1024), c->d_part, 2 * np, c->prm.pjuge, c->d_scal);
        }
    } else {
        const int nmaxp = c->prm.nmaxp;
        for (int done = 0, pass = 0; done < nmaxp; ++pass) {
            const int nit = std::min(c->tb.T, nmaxp - done);
            if (pass == 0) MARK(c, EV_SOR1_START);
            les_status st = launch_sor_tb(c, c->tb, nit, 0, c->prm.pjuge, nmaxp);
            if (st != LES_OK) return st;
            if (pass == 0) MARK(c, EV_SOR1_END);
            // a pass of one iteration cannot stop part-way: no redo launch
            if (nit > 1 && (st = launch_sor_tb(c, c->tb, nit, 1, c->prm.pjuge, nmaxp)) != LES_OK) return st;
            done += nit;
        }
        // an iteration whose FP32 stop test was undecided runs again with
        // exact sums (at most once per step): one more pass, which returns
        // at once when all nmaxp iterations are done or the SOR stopped, and
        // for multi-iteration passes its redo (the repeated iterations may
        // be the ones where the SOR stops)
        if (nmaxp >= 2 && tb_fast_ok(c, c->tb)) {
            les_status st = launch_sor_tb(c, c->tb, c->tb.T, 0, c->prm.pjuge, nmaxp);
            if (st != LES_OK) return st;
            if (c->tb.T > 1 && (st = launch_sor_tb(c, c->tb, c->tb.T, 1, c->prm.pjuge, nmaxp)) != LES_OK) return st;
        }
    }
    MARK(c, EV_SOR_END);
    if (c->ref_outer > 0) {
        les_status st = enqueue_refine(c);
        MARK(c, EV_PAV);
        return st;
    }
    if (c->red_mode & LES_RED_F_PAV) {
        LAUNCH(c, k_seq_sum<2>, dim3(1), dim3(kSeqNT), g, c->F.p, c->d_p2 ? c->d_p2 : c->F.p, 0.0f, c->d_scal);
    } else {
        LAUNCH(c, k_pav_reduce, rg, rb, g, c->F.p, c->d_p2 ? c->d_p2 : c->F.p, c->red_kchunk, c->d_part,
               c->d_scal);
        LAUNCH(c, k_final_pav, dim3(1), dim3(1024), c->d_part, np, c->area, c->d_scal);
    }
    LAUNCH(c, k_pav_adjust, rg, rb, g, c->F.p, c->d_p2 ? c->d_p2 : c->F.p, c->d_scal, c->red_kchunk);
    MARK(c, EV_PAV);
    return LES_OK;
}

// One time step after k_step_begin (main_ocl.f95:264-299).
les_status enqueue_step(les_ctx *c, int n, bool exact_sor) {
    les_status s;
    MARK(c, EV_START);
    if ((s = enqueue_bondv1(c, n, true)) != LES_OK) return s;
    MARK(c, EV_BONDV1);
    if ((s = enqueue_velfg_les(c, true)) != LES_OK) return s;
    if ((s = enqueue_press(c, exact_sor)) != LES_OK) return s;
    LAUNCH(c, k_probe, dim3(1), dim3(1), c->geo, c->F, c->d_scal);
    return LES_OK;
}

les_status check_params(const les_params *p) {
    if (!p) return fail(LES_ERR_BAD_ARG, "params is NULL");
    if (p->ip < 2 || p->jp < 2 || p->kp < 3) return fail(LES_ERR_DIMS, "grid %dx%dx%d too small", p->ip, p->jp, p->kp);
    if (p->inflow_mode == LES_INFLOW_POWER_LAW && p->kp < 78)
        return fail(LES_ERR_DIMS, "bondv1 power-law inflow sets k=1..78 (bondv1.f95:26): kp=%d < 78", p->kp);
    if (p->inflow_mode != LES_INFLOW_POWER_LAW && p->inflow_mode != LES_INFLOW_EXTERNAL)
        return fail(LES_ERR_BAD_ARG, "bad inflow_mode %d", p->inflow_mode);
    if (p->nmaxp < 0) return fail(LES_ERR_BAD_ARG, "nmaxp < 0");
    // set.f95:84-88: the IBM feedback gains bound the time step
    if (((-p->beta - powf(p->beta * p->beta - 2.0f * p->alpha, 0.5f)) / p->alpha) < p->dt)
        return fail(LES_ERR_BAD_ARG, "CHECK parameter alpha beta of IBM method (set.f95:84): dt too large");
    const long long si = ((kOX + p->ip + 3) + 31) / 32 * 32;
    const long long tot = si * (p->jp + 4LL) * (p->kp + 4LL);
    if (tot >= (1LL << 31)) return fail(LES_ERR_DIMS, "grid too large for 32-bit box indexing");
    return LES_OK;
}

// One-iteration passes of this shape may take the FP32 stop test of
// tb_finish_fast: at most 2^16 adds from a term to the root of its sum
// (4 per plane of a k chunk, two block sums of 5 + warps adds, and the
// strided pass over the block partials), a threshold below 2^40, and
// LES_SOR_SUMS not set to "exact".
bool tb_fast_ok(const les_ctx *c, const TbShape &sh) {
    if (sh.T > 2 || !c->sor_fp32_test || !(c->prm.pjuge < 0x1p40f)) return false;
    const int kc = cdiv(c->prm.kp, sh.nch), nt = 32 * tb_warps(sh.T, sh.ty) / sh.rows;
    const long long nblk = (long long)cdiv(c->prm.ip, tb_tx(sh.T)) * cdiv(c->prm.jp, sh.ty) * cdiv(c->prm.kp, kc);
    const long long depth = 4LL * sh.rows * kc + 2 * (5 + nt / 32) + (nblk + nt - 1) / nt;
    return depth <= (1LL << 16);
}

// Launch one temporal-blocked SOR pass (mode 0) or its redo (mode 1); the
// step has itmax iterations.  tuning: read and write only the second p
// buffer (scratch between steps), so timing passes leave the model state
// alone.
les_status launch_sor_tb(les_ctx *c, const TbShape &sh, int niter, int mode, float pjuge, int itmax, bool tuning,
                         const SorBufs *bufs) {
    const int kc = cdiv(c->prm.kp, sh.nch);
    const dim3 grid(cdiv(c->prm.ip, tb_tx(sh.T)), cdiv(c->prm.jp, sh.ty), cdiv(c->prm.kp, kc));
    const dim3 block(32 * tb_warps(sh.T, sh.ty) / sh.rows);
    const size_t sm = tb_smem(sh.T, sh.ty);
    TbArgs a;
    a.pb0 = tuning ? c->d_p2 : c->F.p;
    a.pb1 = c->d_p2;
    a.rhs = c->F.rhs;
    a.cn1k = c->d_tables + c->tl.cn1k;
    a.ty = sh.ty;
    a.kc = kc;
    a.niter = niter;
    a.mode = mode;
    a.itmax = itmax;
    a.fast = (!c->dd && tb_fast_ok(c, sh)) ? 1 : 0;
    a.pjuge = pjuge;
    a.part = c->d_part;
    a.sc = c->d_scal;
    if (bufs) {
        a.pb0 = bufs->pb0;
        a.pb1 = bufs->pb1;
        a.rhs = bufs->rhs;
        a.sc = bufs->sc;
    }
    const Geo &g = c->geo;
#define TBL(TT, KT) LAUNCH_SMEM(c, (k_sor_tb<TT, KT>), grid, block, sm, g, a, c->kq)
    // one-iteration passes: CN1K, odd jp, and DD (a rank of an x-decomposed
    // domain: own-column sums, finished by the host) as template arguments
    const int v1 = (c->cn1_by_k ? 1 : 0) + (c->prm.jp % 2 ? 2 : 0) + (c->dd ? 4 : 0);
#define S1L(K, KT, JO, DDV) LAUNCH_SMEM(c, (K<KT, JO, DDV>), grid, block, s1_smem(sh.ty), g, a, c->kq)
#define S1SW(K)                                         \
    switch (v1) {                                      \
        case 0: S1L(K, false, false, false); break;    \
        case 1: S1L(K, true, false, false); break;     \
        case 2: S1L(K, false, true, false); break;     \
        case 3: S1L(K, true, true, false); break;      \
        case 4: S1L(K, false, false, true); break;     \
        case 5: S1L(K, true, false, true); break;      \
        case 6: S1L(K, false, true, true); break;      \
        default: S1L(K, true, true, true); break;      \
    }
    if (sh.rows == 2) {  // T = 1 (tb_shape_ok)
        S1SW(k_sor1p);
        return LES_OK;
    }
    if (sh.T == 1) {
        S1SW(k_sor1);
        return LES_OK;
    }
#undef S1SW
#undef S1L
    switch (sh.T * 2 + (c->cn1_by_k ? 1 : 0)) {
        case 4: LAUNCH_SMEM(c, k_sor2<false>, grid, block, s2_smem(sh.ty), g, a, c->kq); break;
        case 5: LAUNCH_SMEM(c, k_sor2<true>, grid, block, s2_smem(sh.ty), g, a, c->kq); break;
        case 6: TBL(3, false); break;
        case 7: TBL(3, true); break;
        default: return fail(LES_ERR_BAD_ARG, "SOR pass shape %d,%d", sh.T, sh.ty);
    }
#undef TBL
    return LES_OK;
}

// Largest dynamic shared memory of each pass kernel: the opt-in limit minus
// the kernel's static buffers.
int g_tb_dyn_max = 0;
les_status set_tb_smem_attrs() {
    int dev = 0, optin = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int lim = optin;
#define TBA(TT, KT)                                                                                \
    {                                                                                              \
        cudaFuncAttributes fa;                                                                     \
        CK(cudaFuncGetAttributes(&fa, k_sor_tb<TT, KT>));                                          \
        const int mx = optin - (int)fa.sharedSizeBytes;                                            \
        CK(cudaFuncSetAttribute(k_sor_tb<TT, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)); \
        lim = std::min(lim, mx);                                                                   \
    }
    TBA(3, false) TBA(3, true)
#undef TBA
#define S1A(KT, JO, DDV)                                                                                \
    {                                                                                                   \
        cudaFuncAttributes fa;                                                                          \
        CK(cudaFuncGetAttributes(&fa, k_sor1<KT, JO, DDV>));                                            \
        const int mx = optin - (int)fa.sharedSizeBytes;                                                 \
        CK(cudaFuncSetAttribute(k_sor1<KT, JO, DDV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)); \
        lim = std::min(lim, mx);                                                                   \
    }
    S1A(false, false, false) S1A(true, false, false) S1A(false, true, false) S1A(true, true, false)
    S1A(false, false, true) S1A(true, false, true) S1A(false, true, true) S1A(true, true, true)
#undef S1A
#define S1PA(KT, JO, DDV)                                                                                \
    {                                                                                                    \
        cudaFuncAttributes fa;                                                                           \
        CK(cudaFuncGetAttributes(&fa, k_sor1p<KT, JO, DDV>));                                            \
        const int mx = optin - (int)fa.sharedSizeBytes;                                                  \
        CK(cudaFuncSetAttribute(k_sor1p<KT, JO, DDV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)); \
        lim = std::min(lim, mx);                                                                    \
    }
    S1PA(false, false, false) S1PA(true, false, false) S1PA(false, true, false) S1PA(true, true, false)
    S1PA(false, false, true) S1PA(true, false, true) S1PA(false, true, true) S1PA(true, true, true)
#undef S1PA
#define S2A(KT)                                                                                \
    {                                                                                          \
        cudaFuncAttributes fa;                                                                 \
        CK(cudaFuncGetAttributes(&fa, k_sor2<KT>));                                            \
        const int mx = optin - (int)fa.sharedSizeBytes;                                        \
        CK(cudaFuncSetAttribute(k_sor2<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)); \
        lim = std::min(lim, mx);                                                               \
    }
    S2A(false) S2A(true)
#undef S2A
    g_tb_dyn_max = lim;
    return LES_OK;
}

// Process-wide cache of autotuned SOR pass shapes: (ip, jp, kp, SMs) -> shape.
struct TuneKey {
    int ip, jp, kp, nsm;
    bool operator<(const TuneKey &o) const {
        return std::tie(ip, jp, kp, nsm) < std::tie(o.ip, o.jp, o.kp, o.nsm);
    }
};
std::map<TuneKey, TbShape> g_tune;
std::mutex g_tune_mu;

// A shape this context can launch: it fits the kernel limits, the shared
// memory and the partial-sum array.
bool tb_shape_ok(const les_ctx *c, const TbShape &sh) {
    if (!tb_fits(sh.T, sh.ty) || sh.nch < 1 || sh.nch > kTbMaxChunks) return false;
    if (sh.rows != 1 && (sh.rows != 2 || sh.T != 1 || tb_rh(1, sh.ty) % 2)) return false;
    // odd jp: one iteration per pass (k_sor1), each real row once in a region
    if ((c->prm.jp % 2) != 0 && (sh.T != 1 || tb_rh(1, sh.ty) > c->prm.jp)) return false;
    const size_t smem = sh.T == 1 ? s1_smem(sh.ty) : (sh.T == 2 ? s2_smem(sh.ty) : tb_smem(sh.T, sh.ty));
    if (smem > (size_t)g_tb_dyn_max) return false;
    const int kc = cdiv(c->prm.kp, sh.nch);
    const long long nblk = (long long)cdiv(c->prm.ip, tb_tx(sh.T)) * cdiv(c->prm.jp, sh.ty) * cdiv(c->prm.kp, kc);
    return nblk * kTbTMax <= c->npart;
}

// Autotuner: time each candidate shape on this context's rhs and scratch p
// buffer with CUDA events (two passes after one warm-up pass, the stop test
// disabled; the passes run in place, so the values are meaningless) and
// keep the fastest time per SOR iteration.  Runs once per grid and device;
// LES_SOR_TILE=T,ty[,k chunks] overrides it.  Results persist
// in the file named by LES_TUNE_CACHE.
les_status autotune_sor(les_ctx *c) {
    int dev = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const TuneKey key{c->prm.ip, c->prm.jp, c->prm.kp, nsm};
    TbShape best;
    if (const char *ov = std::getenv("LES_SOR_TILE")) {  // taken where this grid can run it
        std::sscanf(ov, "%d,%d,%d,%d", &best.T, &best.ty, &best.nch, &best.rows);
        if (!tb_shape_ok(c, best)) best = TbShape{};
    }
    if (!best.T) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) best = it->second;
    }
    const char *cache = std::getenv("LES_TUNE_CACHE");
    if (!best.T && cache) {
        if (FILE *fp = std::fopen(cache, "r")) {
            int a, b, cc, d;
            TbShape sh;
            while (std::fscanf(fp, "%d %d %d %d %d %d %d %d", &a, &b, &cc, &d, &sh.T, &sh.ty, &sh.nch, &sh.rows) == 8)
                if (a == key.ip && b == key.jp && cc == key.kp && d == key.nsm) best = sh;
            std::fclose(fp);
        }
    }
    if (!best.T) {
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        double best_t = 0.0;
        // candidates: region heights 8, 12, .., 32 rows, and per (T, k chunks)
        // and wave count w = 1..4 the smallest tile height whose grid still
        // fits in w waves of one CTA per SM (no partly filled last wave)
        std::vector<TbShape> cand;
        for (int T = 1; T <= kTbTMax; ++T)
            for (int nch = 1; nch <= 4; nch *= 2) {
                for (int rh = 8; rh <= 32; rh += 4) cand.push_back(TbShape{T, rh - 2 * tb_ring(T), nch});
                const long long gx = cdiv(c->prm.ip, tb_tx(T));
                for (int w = 1; w <= 4; ++w)
                    for (int ty = 4; ty + 2 * tb_ring(T) <= kTbMaxRH; ++ty)
                        if (gx * cdiv(c->prm.jp, ty) * nch <= (long long)w * nsm) {
                            if ((ty + 2 * tb_ring(T)) % 4) cand.push_back(TbShape{T, ty, nch});
                            break;
                        }
            }
        // and every one-iteration shape with two rows per warp where it has an
        // even region height, with its own wave-fitted heights (even regions)
        for (size_t q = 0, n0 = cand.size(); q < n0; ++q)
            if (cand[q].T == 1 && tb_rh(1, cand[q].ty) % 2 == 0) {
                TbShape s2 = cand[q];
                s2.rows = 2;
                cand.push_back(s2);
            }
        for (int nch = 1; nch <= 4; nch *= 2) {
            const long long gx = cdiv(c->prm.ip, tb_tx(1));
            for (int w = 1; w <= 4; ++w)
                for (int ty = 4; tb_rh(1, ty) <= kTbMaxRH; ty += 2)
                    if (gx * cdiv(c->prm.jp, ty) * nch <= (long long)w * nsm) {
                        if (tb_rh(1, ty) % 4) cand.push_back(TbShape{1, ty, nch, 2});
                        break;
                    }
        }
        for (const TbShape &sh : cand) {
            const int T = sh.T, nch = sh.nch;
            if (sh.ty < 4 || (nch > 1 && cdiv(c->prm.kp, nch) < 8) || !tb_shape_ok(c, sh)) continue;
            CK(cudaMemsetAsync(c->d_scal, 0, sizeof(Scal), c->stream));
            les_status st = launch_sor_tb(c, sh, T, 0, -1.0f, INT_MAX, true);
            if (st != LES_OK) return st;
            CK(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < 2; ++r)
                if ((st = launch_sor_tb(c, sh, T, 0, -1.0f, INT_MAX, true)) != LES_OK) return st;
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            const double per_iter = ms / (2.0 * T);
            if (!best.T || per_iter < best_t) best_t = per_iter, best = sh;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        CK(cudaMemsetAsync(c->d_scal, 0, sizeof(Scal), c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (!best.T) return fail(LES_ERR_DIMS, "no SOR pass shape fits");
        if (cache)
            if (FILE *fp = std::fopen(cache, "a")) {
                std::fprintf(fp, "%d %d %d %d %d %d %d %d\n", key.ip, key.jp, key.kp, key.nsm, best.T, best.ty,
                             best.nch, best.rows);
                std::fclose(fp);
            }
    }
    if (!tb_shape_ok(c, best))
        return fail(LES_ERR_BAD_ARG, "SOR pass shape %d,%d,%d out of range", best.T, best.ty, best.nch);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = best;
    }
    c->tb = best;
    return LES_OK;
}

// True when p's ghosts hold what boundp1 then boundp2 would give
// (boundp.f95:5-44), the state every press ends in.
bool p_ghosts_consistent(const float *p, int ip, int jp, int kp) {
    const size_t ni = ip + 3, nj = jp + 3;
    auto P = [&](int i, int j, int k) { return p[(size_t)i + ni * ((size_t)j + nj * (size_t)k)]; };
    auto same = [](float a, float b) { return std::memcmp(&a, &b, 4) == 0; };
    for (int k = 1; k <= kp; ++k)
        for (int j = 1; j <= jp; ++j)
            if (!same(P(0, j, k), P(1, j, k)) || !same(P(ip + 1, j, k), P(ip, j, k))) return false;
    for (int k = 1; k <= kp; ++k)
        for (int i = 1; i <= ip; ++i)
            if (!same(P(i, 0, k), P(i, jp, k)) || !same(P(i, jp + 1, k), P(i, 1, k))) return false;
    for (int j = 1; j <= jp; ++j)
        for (int i = 1; i <= ip; ++i)
            if (!same(P(i, j, 0), P(i, j, 1)) || !same(P(i, j, kp + 1), P(i, j, kp))) return false;
    return true;
}

}  // namespace

extern "C" {

const char *les_last_error_string(void) { return g_err.c_str(); }

const char *les_version(void) { return "lesb200 0.1 (sm_100a)"; }

les_status les_params_default(les_params *p, int ip, int jp, int kp) {
    LES_RANGE("les_params_default");
    if (!p) return fail(LES_ERR_BAD_ARG, "params is NULL");
    std::memset(p, 0, sizeof *p);
    p->ip = ip;
    p->jp = jp;
    p->kp = kp;
    p->dt = 0.2f;
    p->ro = 1.1763f;
    p->vn = 15.83f * powf(10.0f, -6.0f);
    p->alpha = -10.0f;
    p->beta = -1.0f;
    p->cs0 = 0.1f;
    p->nmaxp = 50;
    p->pjuge = 0.0001f;
    p->omega = 1.0f;
    p->inflow_mode = LES_INFLOW_POWER_LAW;
    p->ical = 0;
    return ok();
}

les_status les_ctx_create(const les_params *prm, les_ctx **out) {
    LES_RANGE("les_ctx_create");
    if (!out) return fail(LES_ERR_BAD_ARG, "out is NULL");
    *out = nullptr;
    les_status s = check_params(prm);
    if (s != LES_OK) return s;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LES_ERR_CUDA, "no CUDA device");
    }
    les_ctx *c = new les_ctx();
    c->prm = *prm;
    if (const char *sums = std::getenv("LES_SOR_SUMS")) c->sor_fp32_test = std::strcmp(sums, "exact") != 0;
    const int ip = prm->ip, jp = prm->jp, kp = prm->kp;
    Geo &g = c->geo;
    g.im = ip;
    g.jm = jp;
    g.km = kp;
    g.olo = 1;
    g.ohi = ip;
    g.ox = kOX;
    g.si = ((kOX + ip + 3) + 31) / 32 * 32;
    g.sj = jp + 4;
    g.sk = kp + 4;
    g.dt = prm->dt;
    g.ro = prm->ro;
    g.vn = prm->vn;
    g.alpha = prm->alpha;
    g.beta = prm->beta;
    g.omega = prm->omega;
    c->box_elems = (size_t)g.si * g.sj * g.sk;
    auto cleanup = [&](les_status st) {
        const std::string msg = g_err;  // destroy resets the error string
        les_ctx_destroy(c);
        g_err = msg;
        return st;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(LES_ERR_CUDA, "cudaStreamCreate failed"));
    if (cudaMalloc(&c->d_fields, sizeof(float) * c->box_elems * LES_NFIELDS) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(fail(LES_ERR_NOMEM, "cannot allocate %.2f GB of fields",
                            sizeof(float) * c->box_elems * LES_NFIELDS / 1e9));
    }
    if (cudaMemsetAsync(c->d_fields, 0, sizeof(float) * c->box_elems * LES_NFIELDS, c->stream) != cudaSuccess)
        return cleanup(fail(LES_ERR_CUDA, "memset fields"));
    c->tl = table_layout(ip, jp, kp);
    if (cudaMalloc(&c->d_tables, sizeof(float) * c->tl.total) != cudaSuccess)
        return cleanup(fail(LES_ERR_NOMEM, "tables"));
    if (cudaMalloc(&c->d_scal, sizeof(Scal)) != cudaSuccess) return cleanup(fail(LES_ERR_NOMEM, "scalars"));
    cudaMemsetAsync(c->d_scal, 0, sizeof(Scal), c->stream);
    // reduction grid: 32x8 blocks over (i,j), k split into chunks of at most
    // 8 planes (short per-thread loops keep many loads in flight)
    c->red_gx = cdiv(ip, kRedBX);
    c->red_gy = cdiv(jp, kRedBY);
    int nk = std::max(cdiv(4 * 148, (long long)c->red_gx * c->red_gy), cdiv(kp, 8));
    nk = nk < 1 ? 1 : (nk > kp ? kp : nk);
    c->red_kchunk = cdiv(kp, nk);
    c->red_nk = cdiv(kp, c->red_kchunk);
    c->npart = 2 * c->red_gx * c->red_gy * c->red_nk;
    if (set_tb_smem_attrs() != LES_OK) return cleanup(LES_ERR_CUDA);
    {
        const int ms = (int)mom_smem(false);
        const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
        if (cudaFuncSetAttribute(k_mom1<true, true>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom1<true, false>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom1<false, false>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<true, true, true>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<true, true, false>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<true, false, false>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<false, true, true>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<false, true, false>, A, ms) != cudaSuccess ||
            cudaFuncSetAttribute(k_mom2<false, false, false>, A, ms) != cudaSuccess)
            return cleanup(fail(LES_ERR_CUDA, "shared memory attribute"));
    }
    // the largest SOR pass grid: narrowest tiles, 4-row tiles, most k chunks
    c->npart = std::max(c->npart, kTbTMax * cdiv(ip, tb_tx(kTbTMax)) * cdiv(jp, 4) * kTbMaxChunks);
    if (cudaMalloc(&c->d_part, sizeof(FixPart) * c->npart) != cudaSuccess)
        return cleanup(fail(LES_ERR_NOMEM, "partials"));
    if (cudaMalloc(&c->d_p2, sizeof(float) * c->box_elems) != cudaSuccess)
        return cleanup(fail(LES_ERR_NOMEM, "second p buffer"));
    cudaMemsetAsync(c->d_p2, 0, sizeof(float) * c->box_elems, c->stream);
    // staging buffer for Fortran-layout arrays: the largest is diu1/diu5
    // (-1:ip+2, 0:jp+2, 0:kp+2) of the per-routine velfg/les entries
    size_t mx = (size_t)(ip + 4) * (jp + 3) * (kp + 3);
    for (int f = 0; f < LES_NFIELDS; ++f) mx = std::max(mx, field_bounds(f, ip, jp, kp).n());
    c->stage_elems = mx;
    if (cudaMalloc(&c->d_stage, sizeof(float) * mx) != cudaSuccess) return cleanup(fail(LES_ERR_NOMEM, "stage"));
    float *base = c->d_tables;
    const TableLayout &t = c->tl;
    g.dx1 = base + t.dx1 + 1;
    g.dy1 = base + t.dy1;
    g.dzn = base + t.dzn + 1;
    g.dzs = base + t.dzs + 1;
    g.dxs = base + t.dxs;
    g.dys = base + t.dys;
    g.cn2l = base + t.cn2l - 1;
    g.cn2s = base + t.cn2s - 1;
    g.cn3l = base + t.cn3l - 1;
    g.cn3s = base + t.cn3s - 1;
    g.cn4l = base + t.cn4l - 1;
    g.cn4s = base + t.cn4s - 1;
    g.cnA = base + t.cnA - 1;
    g.cnB = base + t.cnB - 1;
    g.cnC = base + t.cnC - 1;
    g.smc = base + t.smc - 1;
    g.wind = base + t.wind;
    g.rdx1 = base + t.rdx1 + 1;
    g.rsx = base + t.rsx + 1;
    g.rdy1 = base + t.rdy1;
    g.rsy = base + t.rsy;
    g.rdzn = base + t.rdzn + 1;
    g.rdzs = base + t.rdzs + 1;
    g.rdzn2 = base + t.rdzn2 + 1;
    float **fp[LES_NFIELDS] = {&c->F.u,    &c->F.v,    &c->F.w,    &c->F.p,     &c->F.usum,  &c->F.vsum,  &c->F.wsum,
                               &c->F.f,    &c->F.g,    &c->F.h,    &c->F.fold,  &c->F.gold,  &c->F.hold,  &c->F.rhs,
                               &c->F.sm,   &c->F.amask, &c->F.bmask, &c->F.cmask, &c->F.dmask};
    for (int f = 0; f < LES_NFIELDS; ++f) *fp[f] = field_ptr(c, f);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return cleanup(fail(LES_ERR_CUDA, "sync"));
    *out = c;
    return ok();
}

les_status les_ctx_destroy(les_ctx *c) {
    LES_RANGE("les_ctx_destroy");
    if (!c) return ok();
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &ge : c->graph)
        if (ge) cudaGraphExecDestroy(ge);
    for (auto &gs : c->graph_src)
        if (gs) cudaGraphDestroy(gs);
    for (auto e : c->tev) cudaEventDestroy(e);
    for (auto x : c->extra) cudaFree(x);
    cudaFree(c->d_fields);
    cudaFree(c->d_tables);
    cudaFree(c->d_scal);
    cudaFree(c->d_part);
    cudaFree(c->d_stage);
    cudaFree(c->d_p2);
    cudaFree(c->d_ave);
    cudaFree(c->d_p64);
    cudaFree(c->d_r32);
    cudaFree(c->d_e0);
    cudaFree(c->d_e1);
    cudaFree(c->d_scal2);
    cudaFree(c->d_ref);
    cudaFree(c->d_dpart);
    cudaFree(c->d_refw);
    cudaFree(c->d_r2);
    cudaFree(c->d_drag);
    cudaFree(c->d_dd);
    if (c->dd_ev) cudaEventDestroy(c->dd_ev);
    spec_release(c->spec);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ok();
}

void *les_ctx_stream(les_ctx *c) { return c ? (void *)c->stream : nullptr; }
uint64_t les_ctx_launch_count(les_ctx *c) { return c ? c->launches : 0; }

les_status les_ctx_field(les_ctx *c, int field, float **dptr, int *ox, int *si, int *sj, int *sk) {
    LES_RANGE("les_ctx_field");
    if (!c || field < 0 || field >= LES_NFIELDS) return fail(LES_ERR_BAD_ARG, "bad field");
    if (dptr) *dptr = field_ptr(c, field);
    if (ox) *ox = c->geo.ox;
    if (si) *si = c->geo.si;
    if (sj) *sj = c->geo.sj;
    if (sk) *sk = c->geo.sk;
    return ok();
}

static les_status upload_field(les_ctx *c, int f, const float *host) {
    if (!host) return LES_OK;
    const FBounds b = field_bounds(f, c->prm.ip, c->prm.jp, c->prm.kp);
    CK(cudaMemcpyAsync(c->d_stage, host, sizeof(float) * b.n(), cudaMemcpyHostToDevice, c->stream));
    LAUNCH(c, k_f2box, dim3(cdiv((long long)b.n(), 256 * 4)), dim3(256), c->geo, field_ptr(c, f), c->d_stage, b.li,
           b.lj, b.lk, b.ni(), b.nj(), b.nk());
    return LES_OK;
}

static les_status download_field(les_ctx *c, int f, float *host) {
    if (!host) return LES_OK;
    const FBounds b = field_bounds(f, c->prm.ip, c->prm.jp, c->prm.kp);
    // rhs is kept before the rhsav subtraction; the caller gets
    // rhs - rhsav on the interior as press.f95:139-145 leaves it.
    const bool sub = (f == LES_F_RHS) && c->rhs_raw;
    float rhsav = 0.0f;
    if (sub) {
        Scal sc;
        CK(cudaMemcpyAsync(&sc, c->d_scal, sizeof sc, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        rhsav = sc.rhsav;
    }
    LAUNCH(c, k_box2f, dim3(cdiv((long long)b.n(), 256 * 4)), dim3(256), c->geo, field_ptr(c, f), c->d_stage, b.li,
           b.lj, b.lk, b.ni(), b.nj(), b.nk(), rhsav, sub ? 1 : 0);
    CK(cudaMemcpyAsync(host, c->d_stage, sizeof(float) * b.n(), cudaMemcpyDeviceToHost, c->stream));
    return LES_OK;
}

// Index of the first non-finite float in a[0..n), or -1.  Chunks are
// OR-reduced without branches (vectorisable); only a hit is located.
static long long first_non_finite(const float *a, size_t n) {
    const uint32_t *b = reinterpret_cast<const uint32_t *>(a);
    constexpr size_t kChunk = 4096;
    for (size_t o = 0; o < n; o += kChunk) {
        const size_t e = std::min(n, o + kChunk);
        uint32_t hit = 0;
        for (size_t t = o; t < e; ++t) hit |= (uint32_t)((b[t] & 0x7f800000u) == 0x7f800000u);
        if (hit)
            for (size_t t = o; t < e; ++t)
                if ((b[t] & 0x7f800000u) == 0x7f800000u) return (long long)t;
    }
    return -1;
}

// Input check of les_ctx_upload: every array given must be finite (the
// reference has no such check; a NaN or Inf would spread through the step).
static les_status scan_inputs(les_ctx *c, const les_host_fields *hf) {
    const int ip = c->prm.ip, jp = c->prm.jp, kp = c->prm.kp;
    struct Arr {
        const char *name;
        const float *p;
        size_t n;
    };
    const Arr tabs[] = {{"dx1", hf->dx1, (size_t)ip + 3},  {"dy1", hf->dy1, (size_t)jp + 2},
                        {"dzn", hf->dzn, (size_t)kp + 4},  {"dzs", hf->dzs, (size_t)kp + 4},
                        {"dxs", hf->dxs, (size_t)ip + 1},  {"dys", hf->dys, (size_t)jp + 1},
                        {"cn2l", hf->cn2l, (size_t)ip},    {"cn2s", hf->cn2s, (size_t)ip},
                        {"cn3l", hf->cn3l, (size_t)jp},    {"cn3s", hf->cn3s, (size_t)jp},
                        {"cn4l", hf->cn4l, (size_t)kp},    {"cn4s", hf->cn4s, (size_t)kp},
                        {"z2", hf->z2, (size_t)kp + 2},    {"wind_profile", hf->wind_profile, (size_t)jp * kp}};
    for (const Arr &a : tabs) {
        if (!a.p) continue;
        const long long t = first_non_finite(a.p, a.n);
        if (t >= 0) return fail(LES_ERR_NAN, "les_ctx_upload: %s[%lld] is not finite", a.name, t);
    }
    static const char *names[LES_NFIELDS] = {"u",    "v",    "w",    "p",      "usum",   "vsum",   "wsum",
                                             "f",    "g",    "h",    "fold",   "gold",   "hold",   "rhs",
                                             "sm",   "amask1", "bmask1", "cmask1", "dmask1"};
    const float *src[LES_NFIELDS] = {hf->u,    hf->v,    hf->w,    hf->p,   hf->usum,   hf->vsum,   hf->wsum,
                                     hf->f,    hf->g,    hf->h,    hf->fold, hf->gold,  hf->hold,   hf->rhs,
                                     hf->sm,   hf->amask1, hf->bmask1, hf->cmask1, hf->dmask1};
    for (int f = 0; f < LES_NFIELDS; ++f) {
        if (!src[f]) continue;
        const FBounds b = field_bounds(f, ip, jp, kp);
        const long long t = first_non_finite(src[f], b.n());
        if (t >= 0) {
            const int i = b.li + (int)(t % b.ni()), r = (int)(t / b.ni());
            const int j = b.lj + r % b.nj(), k = b.lk + r / b.nj();
            return fail(LES_ERR_NAN, "les_ctx_upload: %s(%d,%d,%d) is not finite", names[f], i, j, k);
        }
    }
    return LES_OK;
}

les_status les_ctx_upload(les_ctx *c, const les_host_fields *hf) {
    LES_RANGE("les_ctx_upload");
    if (!c || !hf) return fail(LES_ERR_BAD_ARG, "NULL argument");
    if (!hf->dx1 || !hf->dy1 || !hf->dzn || !hf->dzs || !hf->dxs || !hf->dys || !hf->cn2l || !hf->cn2s ||
        !hf->cn3l || !hf->cn3s || !hf->cn4l || !hf->cn4s)
        return fail(LES_ERR_BAD_ARG, "metric tables and Poisson coefficients are required");
    les_status s = scan_inputs(c, hf);
    if (s != LES_OK) return s;
    s = build_tables(c, hf, true);
    if (s != LES_OK) return s;
    const float *src[LES_NFIELDS] = {hf->u,    hf->v,    hf->w,    hf->p,   hf->usum,   hf->vsum,   hf->wsum,
                                     hf->f,    hf->g,    hf->h,    hf->fold, hf->gold,  hf->hold,   hf->rhs,
                                     hf->sm,   hf->amask1, hf->bmask1, hf->cmask1, hf->dmask1};
    for (int f = 0; f < LES_NFIELDS; ++f)
        if ((s = upload_field(c, f, src[f])) != LES_OK) return s;
    // cn1 is rebuilt from its separable parts in the SOR kernel; a caller's
    // cn1 must equal init.f95:87-93 bit for bit.
    if (hf->cn1) {
        const int ip = c->prm.ip, jp = c->prm.jp, kp = c->prm.kp;
        const std::vector<float> &h = c->h_tables;
        for (int k = 1; k <= kp; ++k)
            for (int j = 1; j <= jp; ++j)
                for (int i = 1; i <= ip; ++i) {
                    const float want = 1.0f / (h[c->tl.cnA + i - 1] + h[c->tl.cnB + j - 1] + h[c->tl.cnC + k - 1]);
                    const float got = hf->cn1[(size_t)(i - 1) + (size_t)ip * ((j - 1) + (size_t)jp * (k - 1))];
                    if (std::memcmp(&want, &got, 4) != 0)
                        return fail(LES_ERR_BAD_ARG,
                                    "cn1(%d,%d,%d) differs from 1/(2/(dxs*dxs)+2/(dys*dys)+2/(dzs*dzs)) (init.f95:87-93)",
                                    i, j, k);
                }
    }
    CK(cudaStreamSynchronize(c->stream));
    c->uploaded = true;
    c->rhs_raw = false;
    c->p_ghosts_ok = hf->p ? p_ghosts_consistent(hf->p, c->prm.ip, c->prm.jp, c->prm.kp) : false;
    return ok();
}

les_status les_ctx_download(les_ctx *c, les_host_fields *hf) {
    LES_RANGE("les_ctx_download");
    if (!c || !hf) return fail(LES_ERR_BAD_ARG, "NULL argument");
    float *dst[LES_NFIELDS] = {hf->u,  hf->v,  hf->w,    hf->p,    hf->usum, hf->vsum,   hf->wsum,
                               hf->f,  hf->g,  hf->h,    hf->fold, hf->gold, hf->hold,   hf->rhs,
                               hf->sm, hf->amask1, hf->bmask1, hf->cmask1, hf->dmask1};
    les_status s;
    for (int f = 0; f < LES_NFIELDS; ++f) {
        if ((s = download_field(c, f, dst[f])) != LES_OK) return s;
        CK(cudaStreamSynchronize(c->stream));
    }
    if (hf->delx1) {
        for (int k = 1; k <= c->prm.kp; ++k) {
            const float *h = c->h_tables.data();
            hf->delx1[k - 1] = powf(h[c->tl.dx1 + 1] * h[c->tl.dy1] * h[c->tl.dzn + k + 1], 1.0f / 3.0f);
        }
    }
    return ok();
}

les_status les_ctx_field_sums(les_ctx *c, double *sums) {
    LES_RANGE("les_ctx_field_sums");
    if (!c || !sums) return fail(LES_ERR_BAD_ARG, "NULL argument");
    double *d_out = reinterpret_cast<double *>(c->d_stage);  // LES_NFIELDS doubles
    for (int f = 0; f < LES_NFIELDS; ++f) {
        const FBounds b = field_bounds(f, c->prm.ip, c->prm.jp, c->prm.kp);
        const bool sub = (f == LES_F_RHS) && c->rhs_raw;
        const int nb = (int)std::min<long long>(cdiv((long long)b.n(), kRedNT * 8LL), (long long)c->npart);
        LAUNCH(c, k_field_sum, dim3(nb), dim3(kRedNT), c->geo, field_ptr(c, f), b.li, b.lj, b.lk, b.ni(), b.nj(),
               b.nk(), c->d_scal, sub ? 1 : 0, c->d_part);
        LAUNCH(c, k_field_sum_final, dim3(1), dim3(1024), c->d_part, nb, d_out + f);
    }
    CK(cudaMemcpyAsync(sums, d_out, sizeof(double) * LES_NFIELDS, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ok();
}

les_status les_ctx_warmup(les_ctx *c, int n) {
    LES_RANGE("les_ctx_warmup");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    if (!c->uploaded) return fail(LES_ERR_STATE, "warmup before upload");
    les_status s;
    LAUNCH(c, k_step_begin, dim3(1), dim3(1), c->d_scal, n);
    LAUNCH(c, k_zero_fgh, dim3(cdiv((long long)(c->prm.ip + 1) * (c->prm.jp + 1) * (c->prm.kp + 1), 1024)), dim3(256),
           c->geo, c->F);
    if ((s = enqueue_bondv1(c, n, false)) != LES_OK) return s;
    if ((s = enqueue_boundp(c, false)) != LES_OK) return s;
    if ((s = enqueue_velfg_les(c, false)) != LES_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    c->p_ghosts_ok = true;  // ifdata.f95:260-262 applied boundp1, boundp2
    return ok();
}

les_status les_ctx_sor_tile(les_ctx *c, int *T, int *ty) {
    LES_RANGE("les_ctx_sor_tile");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    if (T) *T = c->tb.T;
    if (ty) *ty = c->tb.ty;
    return ok();
}

les_status les_ctx_sor_shape(les_ctx *c, int *T, int *ty, int *tx, int *nch) {
    LES_RANGE("les_ctx_sor_shape");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    if (T) *T = c->tb.T;
    if (ty) *ty = c->tb.ty;
    if (tx) *tx = c->tb.T ? tb_tx(c->tb.T) : 0;
    if (nch) *nch = c->tb.nch;
    return ok();
}

les_status les_ctx_sor_rows(les_ctx *c, int *rows) {
    LES_RANGE("les_ctx_sor_rows");
    if (!c || !rows) return fail(LES_ERR_BAD_ARG, "NULL argument");
    *rows = c->tb.T ? c->tb.rows : 0;
    return ok();
}

float les_ctx_sor_iters_per_launch(les_ctx *c) {
    if (!c) return 0.0f;
    const bool exact = sor_per_colour(c);
    return exact ? 0.5f : (float)(c->tb.T ? c->tb.T : 2);
}

les_status les_ctx_set_sor_path(les_ctx *c, int exact) {
    LES_RANGE("les_ctx_set_sor_path");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    c->force_exact_sor = exact != 0;
    return ok();
}

les_status les_bounds_violations(unsigned long long *count, int *first_ijk) {
    LES_RANGE("les_bounds_violations");
#ifdef LES_CHECKED
    LesOob h{};
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpyFromSymbol(&h, g_les_oob, sizeof h));
    if (count) *count = h.count;
    if (first_ijk)
        for (int q = 0; q < 3; ++q) first_ijk[q] = h.claimed ? h.first[q] : 0;
    return ok();
#else
    (void)count;
    (void)first_ijk;
    return fail(LES_ERR_STATE, "not a LES_CHECKED build (liblesb200_checked.so)");
#endif
}

les_status les_ctx_set_reduction_mode(les_ctx *c, int mode) {
    LES_RANGE("les_ctx_set_reduction_mode");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    if (mode < 0 || mode > LES_RED_FAITHFUL) return fail(LES_ERR_BAD_ARG, "bad reduction mode %d", mode);
    if (mode != LES_RED_CANONICAL && c->ref_outer > 0)
        return fail(LES_ERR_STATE, "reference-order sums and the FP64-refined press exclude each other");
    if ((mode & LES_RED_F_SOR) && !c->d_r2) {
        if (cudaMalloc(&c->d_r2, sizeof(float) * c->box_elems) != cudaSuccess) {
            cudaGetLastError();
            return fail(LES_ERR_NOMEM, "reltmp^2 buffer");
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    c->red_mode = mode;
    drop_step_graphs(c);  // the captured steps hold the previous mode's kernels
    return ok();
}

les_status les_set_wind_profile(les_ctx *c, const float *wp) {
    LES_RANGE("les_set_wind_profile");
    if (!c || !wp) return fail(LES_ERR_BAD_ARG, "NULL argument");
    if (c->prm.inflow_mode != LES_INFLOW_EXTERNAL) return fail(LES_ERR_STATE, "context uses the power-law inflow");
    const long long bad = first_non_finite(wp, (size_t)c->prm.jp * c->prm.kp);
    if (bad >= 0) return fail(LES_ERR_NAN, "les_set_wind_profile: wind_profile[%lld] is not finite", bad);
    CK(cudaMemcpyAsync(c->d_tables + c->tl.wind, wp, sizeof(float) * (size_t)c->prm.jp * c->prm.kp,
                       cudaMemcpyHostToDevice, c->stream));
    return ok();
}

les_status les_step(les_ctx *c, int n0, int nsteps) {
    LES_RANGE("les_step");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    if (!c->uploaded) return fail(LES_ERR_STATE, "step before upload");
    if (nsteps < 0) return fail(LES_ERR_BAD_ARG, "nsteps < 0");
    if (c->dd) return fail(LES_ERR_STATE, "a rank of a decomposed domain steps by les_dd_phase");
    for (int s = 0; s < nsteps; ++s) {
        LES_RANGE("step");
        const int n = n0 + s;
        const bool exact = sor_per_colour(c);
        const int gi = ((n == 1 && c->prm.ical == 0) ? 1 : 0) + (exact ? 2 : 0);
        if ((!exact || c->ref_outer > 0) && c->tb.T == 0) {  // the refined press uses the passes too
            LES_RANGE("sor_autotune");
            les_status st = autotune_sor(c);
            if (st != LES_OK) return st;
        }
        if (!c->graph[gi]) {
            // Capture the step once per kind (n==1 broadcast or not); the
            // kernels only see n through that distinction.
            LES_RANGE("step_graph_capture");
            const uint64_t before = c->launches;
            c->capturing_timed = c->tslots > 0;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            les_status st = enqueue_step(c, (gi & 1) ? 1 : 2, exact);
            cudaGraph_t gr = nullptr;
            cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
            c->capturing_timed = false;
            c->graph_kernels[gi] = c->launches - before;
            c->launches = before;  // capturing runs nothing
            if (st != LES_OK) {
                if (gr) cudaGraphDestroy(gr);
                return st;
            }
            if (e != cudaSuccess) return fail(LES_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(&c->graph[gi], gr, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(gr);
                return fail(LES_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
            }
            c->graph_src[gi] = gr;
            c->tnode[gi].clear();
            c->tnode_idx[gi].clear();
            if (c->tslots > 0) {  // find the event record nodes and which event each records
                size_t nn = 0;
                CK(cudaGraphGetNodes(gr, nullptr, &nn));
                std::vector<cudaGraphNode_t> nodes(nn);
                CK(cudaGraphGetNodes(gr, nodes.data(), &nn));
                for (auto nd : nodes) {
                    cudaGraphNodeType ty;
                    CK(cudaGraphNodeGetType(nd, &ty));
                    if (ty != cudaGraphNodeTypeEventRecord) continue;
                    cudaEvent_t ev;
                    CK(cudaGraphEventRecordNodeGetEvent(nd, &ev));
                    for (int w = 0; w < LES_NTEV; ++w)
                        if (ev == c->tev[w]) {
                            c->tnode[gi].push_back(nd);
                            c->tnode_idx[gi].push_back(w);
                        }
                }
            }
        }
        if (c->tslots > 0) {
            const int slot = c->tslot < c->tslots ? c->tslot : c->tslots - 1;
            for (size_t q = 0; q < c->tnode[gi].size(); ++q)
                CK(cudaGraphExecEventRecordNodeSetEvent(c->graph[gi], c->tnode[gi][q],
                                                        c->tev[(size_t)slot * LES_NTEV + c->tnode_idx[gi][q]]));
            if (c->tslot < c->tslots) ++c->tslot;
        }
        LAUNCH(c, k_step_begin, dim3(1), dim3(1), c->d_scal, n);
        CK(cudaGraphLaunch(c->graph[gi], c->stream));
        c->launches += c->graph_kernels[gi];
        c->last_n = n;
        c->rhs_raw = true;
        c->p_ghosts_ok = true;  // press ends with boundp1/boundp2
    }
    return ok();
}

les_status les_ctx_set_timing(les_ctx *c, int nslots) {
    LES_RANGE("les_ctx_set_timing");
    if (!c || nslots < 0) return fail(LES_ERR_BAD_ARG, "bad argument");
    CK(cudaStreamSynchronize(c->stream));
    if (nslots > 0 && c->tslots > 0 && (size_t)nslots * LES_NTEV <= c->tev.size()) {
        c->tslots = nslots;  // re-arm: the pool and the captured graphs stay
        c->tslot = 0;
        return ok();
    }
    // graphs are re-captured with (or without) event nodes for the new pool
    for (int gi = 0; gi < 4; ++gi) {
        if (c->graph[gi]) cudaGraphExecDestroy(c->graph[gi]);
        if (c->graph_src[gi]) cudaGraphDestroy(c->graph_src[gi]);
        c->graph[gi] = nullptr;
        c->graph_src[gi] = nullptr;
    }
    for (auto e : c->tev) cudaEventDestroy(e);
    c->tev.assign((size_t)nslots * LES_NTEV, nullptr);
    for (auto &e : c->tev) CK(cudaEventCreate(&e));
    c->tslots = nslots;
    c->tslot = 0;
    return ok();
}

les_status les_ctx_phase_times(les_ctx *c, int slot, float *ms, int n) {
    LES_RANGE("les_ctx_phase_times");
    if (!c || !ms || slot < 0 || slot >= c->tslots) return fail(LES_ERR_BAD_ARG, "bad slot");
    CK(cudaStreamSynchronize(c->stream));
    // ms[0..7]: consecutive phases between the events; ms[8]: whole step
    for (int w = 0; w < LES_NTEV && w < n; ++w) {
        const int a = (w == LES_NTEV - 1) ? EV_START : w, b = (w == LES_NTEV - 1) ? EV_PAV : w + 1;
        CK(cudaEventElapsedTime(&ms[w], c->tev[(size_t)slot * LES_NTEV + a], c->tev[(size_t)slot * LES_NTEV + b]));
    }
    return ok();
}

les_status les_ctx_sync(les_ctx *c) {
    LES_RANGE("les_ctx_sync");
    if (!c) return fail(LES_ERR_BAD_ARG, "NULL ctx");
    CK(cudaStreamSynchronize(c->stream));
    return ok();
}

les_status les_last_metrics(les_ctx *c, les_metrics *m) {
    LES_RANGE("les_last_metrics");
    if (!c || !m) return fail(LES_ERR_BAD_ARG, "NULL argument");
    Scal s;
    CK(cudaMemcpyAsync(&s, c->d_scal, sizeof s, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    m->n = s.n;
    m->sor_iters = s.sor_iters;
    m->sor = s.sor;
    m->rhsav = s.rhsav;
    m->pav = s.pav;
    m->uout = s.uout;
    m->p_centre = s.probe[0];
    m->u_centre = s.probe[1];
    m->v_centre = s.probe[2];
    m->w_centre = s.probe[3];
    return ok();
}

// ---- context halo (TEMPL:111-127, LES_combined_kernel.cl:345-364) ----
static bool ctx_halo_view(les_ctx *c, int which, CombView &cv, HaloDims &d) {
    const int ip = c->prm.ip, jp = c->prm.jp, kp = c->prm.kp;
    std::memset(&cv, 0, sizeof cv);
    int ext[3] = {0, 0, 0}, vdim = 1;
    Fields &F = c->F;
    switch (which) {
        case LES_H_P:  // p2 = float2(p, p), (0:ip+2,0:jp+2,0:kp+1)
            cv.comp[0] = F.p;
            cv.comp[1] = F.p;
            vdim = 2;
            ext[0] = ip + 3, ext[1] = jp + 3, ext[2] = kp + 2;
            cv.li = 0, cv.lj = 0, cv.lk = 0;
            break;
        case LES_H_UVW:  // float4(u,v,w,0), (0:ip+1,-1:jp+1,-1:kp+1); u,v start at k=0
            cv.comp[0] = F.u, cv.comp[1] = F.v, cv.comp[2] = F.w;
            cv.klo[0] = 0, cv.klo[1] = 0, cv.klo[2] = -1, cv.klo[3] = -1;
            vdim = 4;
            ext[0] = ip + 2, ext[1] = jp + 3, ext[2] = kp + 3;
            cv.li = 0, cv.lj = -1, cv.lk = -1;
            break;
        case LES_H_UVWSUM:
        case LES_H_FGH:
            if (which == LES_H_UVWSUM)
                cv.comp[0] = F.usum, cv.comp[1] = F.vsum, cv.comp[2] = F.wsum;
            else
                cv.comp[0] = F.f, cv.comp[1] = F.g, cv.comp[2] = F.h;
            vdim = 4;
            ext[0] = ip + 1, ext[1] = jp + 1, ext[2] = kp + 1;
            break;
        case LES_H_FGH_OLD:
            cv.comp[0] = F.fold, cv.comp[1] = F.gold, cv.comp[2] = F.hold;
            vdim = 4;
            ext[0] = ip, ext[1] = jp, ext[2] = kp;
            cv.li = 1, cv.lj = 1, cv.lk = 1;
            break;
        case LES_H_RHS:
            cv.comp[0] = F.rhs;
            ext[0] = ip + 2, ext[1] = jp + 2, ext[2] = kp + 2;
            break;
        case LES_H_SM:
            cv.comp[0] = F.sm;
            ext[0] = ip + 3, ext[1] = jp + 3, ext[2] = kp + 2;
            cv.li = -1, cv.lj = -1, cv.lk = 0;
            break;
        default: return false;
    }
    if (which != LES_H_UVW)
        for (int v = 0; v < 4; ++v) cv.klo[v] = cv.lk;
    d = halo_dims(ext[0], ext[1], ext[2], 1, vdim, 0);
    return true;
}

size_t les_ctx_halo_floats(les_ctx *c, int which) {
    CombView cv;
    HaloDims d;
    if (!c || !ctx_halo_view(c, which, cv, d)) return 0;
    return d.vsz * d.vdim;
}

static les_status ctx_halo(les_ctx *c, int which, float *buf, int write) {
    CombView cv;
    HaloDims d;
    if (!c || !buf) return fail(LES_ERR_BAD_ARG, "NULL argument");
    if (!ctx_halo_view(c, which, cv, d)) return fail(LES_ERR_BAD_ARG, "bad halo id %d", which);
    const size_t n = d.vsz * d.vdim;
    if (n > c->stage_elems) return fail(LES_ERR_DIMS, "halo larger than the staging buffer");
    // p2 = (p, p): both components read p; on write the second is ignored,
    // so one value lands on each p point
    if (write && which == LES_H_P) cv.comp[1] = nullptr;
    // page-locked host memory (cudaHostAlloc / cudaHostRegister) is mapped
    // into the device's address space: the kernel reads or writes the
    // caller's buffer across the host link itself, with no staging copy
    cudaPointerAttributes pa{};
    float *mapped = nullptr;
    if (cudaPointerGetAttributes(&pa, buf) == cudaSuccess) {
        if (pa.type == cudaMemoryTypeHost && pa.devicePointer) mapped = static_cast<float *>(pa.devicePointer);
    } else {
        cudaGetLastError();
    }
    if (mapped) {
        LAUNCH(c, k_ctx_halo, dim3(cdiv((long long)n, 256)), dim3(256), c->geo, cv, mapped, d, write);
    } else {
        if (write) CK(cudaMemcpyAsync(c->d_stage, buf, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
        LAUNCH(c, k_ctx_halo, dim3(cdiv((long long)n, 256)), dim3(256), c->geo, cv, c->d_stage, d, write);
        if (!write) CK(cudaMemcpyAsync(buf, c->d_stage, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return ok();
}
les_status les_ctx_halo_read(les_ctx *c, int which, float *buf) {
    LES_RANGE("les_ctx_halo_read");
    return ctx_halo(c, which, buf, 0);
}
les_status les_ctx_halo_write(les_ctx *c, int which, const float *buf) {
    LES_RANGE("les_ctx_halo_write");
    return ctx_halo(c, which, const_cast<float *>(buf), 1);
}

}  // extern "C"

#include "les_routines_api.inc"
#include "les_stats_io.inc"
#include "les_ensemble.inc"
#include "les_refine.inc"
#include "les_adjoint.inc"
#include "les_adjstep.inc"
#include "les_dd.inc"
