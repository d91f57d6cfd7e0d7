// les_oracle.cpp -- CPU restatement of the LES_Halo Fortran time step.
//
// TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; see les_oracle.h).
// Each routine follows the reference file and line range named above it, with
// the same loop bounds, the same in-place update order and the same IEEE
// single-precision expression order.  Build with -ffp-contract=off.
#include "les_oracle.h"

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Fortran column-major array view with arbitrary lower bounds.
struct A3 {
    float *a;
    int li, lj, lk, ni, nj, nk;
    inline float &operator()(int i, int j, int k) const {
#ifdef ORACLE_CHECK
        if (i < li || i >= li + ni || j < lj || j >= lj + nj || k < lk || k >= lk + nk) {
            std::fprintf(stderr, "oracle: index (%d,%d,%d) outside [%d:%d,%d:%d,%d:%d]\n", i, j, k,
                         li, li + ni - 1, lj, lj + nj - 1, lk, lk + nk - 1);
            std::abort();
        }
#endif
        return a[(size_t)(i - li) + (size_t)ni * ((size_t)(j - lj) + (size_t)nj * (size_t)(k - lk))];
    }
};
struct A1 {
    float *a;
    int l;
    inline float &operator()(int i) const { return a[i - l]; }
};

inline A3 mk(const float *p, int li, int ui, int lj, int uj, int lk, int uk) {
    return A3{const_cast<float *>(p), li, lj, lk, ui - li + 1, uj - lj + 1, uk - lk + 1};
}
inline A1 mk1(const float *p, int l) { return A1{const_cast<float *>(p), l}; }

// Array shapes of main_ocl.f95:41-167 with ip=im, jp=jm, kp=km.
#define ARR_U(p) mk(p, 0, ip + 1, -1, jp + 1, 0, kp + 1)
#define ARR_W(p) mk(p, 0, ip + 1, -1, jp + 1, -1, kp + 1)
#define ARR_P(p) mk(p, 0, ip + 2, 0, jp + 2, 0, kp + 1)
#define ARR_F(p) mk(p, 0, ip, 0, jp, 0, kp)
#define ARR_I(p) mk(p, 1, ip, 1, jp, 1, kp)
#define ARR_RHS(p) mk(p, 0, ip + 1, 0, jp + 1, 0, kp + 1)
#define ARR_SM(p) mk(p, -1, ip + 1, -1, jp + 1, 0, kp + 1)
#define ARR_D15(p) mk(p, -1, ip + 2, 0, jp + 2, 0, kp + 2)
#define ARR_D(p) mk(p, 0, ip + 2, 0, jp + 2, 0, kp + 2)
#define ARR_AM(p) mk(p, 0, ip + 1, 0, jp + 1, 0, kp + 1)
#define ARR_BM(p) mk(p, -1, ip + 1, 0, jp + 1, 0, kp + 1)
#define ARR_CM(p) mk(p, 0, ip + 1, -1, jp + 1, 0, kp + 1)
#define ARR_DFU(p) mk(p, 0, ip, 1, jp, 1, kp)
#define ARR_DFV(p) mk(p, 1, ip, 0, jp, 1, kp)

int g_red_mode = ORACLE_RED_CANONICAL;
float g_last_uout = 0.0f;
// FP64-refined press (oracle_set_press_refine): settings and last report
int g_ref_outer = 0, g_ref_inner = 0;
double g_ref_tol = 0.0;
double g_ref_out[4] = {0, 0, 0, 0};  // rhsav, pav, rel_initial, rel_final
int g_ref_done = 0;

// ---------------------------------------------------------------------------
// Canonical global sum (shared definition with the CUDA kernels).
// Each FP32 term x is converted exactly to a signed Q63.64 fixed-point
// integer, truncating toward zero below 2^-64; the integers are summed
// exactly in 128 bits (so the result does not depend on summation order);
// the total T is turned into a double as (double)hi * 2^64 + (double)lo with
// hi = T >> 64 (signed) and lo = T mod 2^64 (unsigned), then scaled by 2^-64.
// Terms that are not finite or have |x| >= 2^62 mark the sum as NaN.
// ---------------------------------------------------------------------------
typedef __int128 i128;

struct FixSum {
    i128 acc = 0;
    bool bad = false;
    void add(float x) {
        uint32_t b;
        std::memcpy(&b, &x, 4);
        const int e = (int)((b >> 23) & 0xffu);
        if (e == 255) { bad = true; return; }
        if (e == 0) return;  // zero or subnormal: below 2^-126, truncates to 0
        const int E = e - 127;
        if (E >= 62) { bad = true; return; }
        const uint64_t mant = (uint64_t)((b & 0x7fffffu) | 0x800000u);
        const int sh = E + 41;  // value * 2^64 = mant * 2^(E-23+64)
        i128 m;
        if (sh >= 0) m = (i128)mant << sh;
        else if (sh > -64) m = (i128)(mant >> (-sh));
        else m = 0;
        acc += (b >> 31) ? -m : m;
    }
    double value() const {
        if (bad) return std::nan("");
        const int64_t hi = (int64_t)(acc >> 64);
        const uint64_t lo = (uint64_t)acc;
        const double two64 = 18446744073709551616.0;
        return ((double)hi * two64 + (double)lo) / two64;
    }
};

template <class F>
double canonical_sum3(int im, int jm, int km, F x) {
    FixSum s;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) s.add(x(i, j, k));
    return s.value();
}

}  // namespace

extern "C" {

void oracle_set_reduction_mode(int mode) { g_red_mode = mode; }
void oracle_set_press_refine(int outer, int inner, double tol) {
    g_ref_outer = outer;
    g_ref_inner = inner;
    g_ref_tol = tol;
}
int oracle_last_refine(double *out4) {
    for (int q = 0; q < 4; ++q) out4[q] = g_ref_out[q];
    return g_ref_done;
}
int oracle_get_reduction_mode(void) { return g_red_mode; }
float oracle_last_uout(void) { return g_last_uout; }

double oracle_canonical_sum(int im, int jm, int km, const float *vals) {
    A3 x = mk(vals, 1, im, 1, jm, 1, km);
    return canonical_sum3(im, jm, km, [&](int i, int j, int k) { return x(i, j, k); });
}

// set.f95:78-82
void oracle_constants(float *ro, float *vn, float *alpha, float *beta) {
    *ro = 1.1763f;
    *vn = 15.83f * std::pow(10.0f, -6.0f);
    *alpha = -10.0f;
    *beta = -1.0f;
}

// grid.f95:55-82 (metric derivation; the dz profile itself is an input).
void oracle_grid_metrics(int ip, int jp, int kp, float *dx1_, float *dxl_, float *dy1_,
                         float *dyl_, float *z2_, float *dzn_, float *dzs_, float *dxs_,
                         float *dys_) {
    A1 dx1 = mk1(dx1_, -1), dxl = mk1(dxl_, 0), dy1 = mk1(dy1_, 0), dyl = mk1(dyl_, 0);
    A1 z2 = mk1(z2_, 1), dzn = mk1(dzn_, -1), dzs = mk1(dzs_, -1), dxs = mk1(dxs_, 0),
       dys = mk1(dys_, 0);
    dxl(0) = 0.0f;
    for (int i = 1; i <= ip; ++i) dxl(i) = dxl(i - 1) + dx1(i);
    dyl(0) = 0.0f;
    for (int j = 1; j <= jp; ++j) dyl(j) = dyl(j - 1) + dy1(j);
    // grid.f95:42-54 sets z2(1) = dzn(1) = 2.5 for its grid; a given dz
    // profile starts at z2(1) = dzn(1).  z2(0) is out of bounds in the
    // reference (it writes the element before z2) and is not kept here.
    z2(1) = dzn(1);
    dzn(kp + 2) = 0.0f;  // not yet set when grid.f95:55 reads it
    for (int k = 2; k <= kp + 2; ++k) z2(k) = z2(k - 1) + dzn(k);
    dzn(kp + 1) = dzn(kp);
    dzn(kp + 2) = dzn(kp + 1);
    dzn(0) = dzn(1);
    dzn(-1) = dzn(0);
    for (int k = 0; k <= kp; ++k) dzs(k) = dzn(k + 1) / 2.0f + dzn(k) / 2.0f;
    for (int i = 0; i <= ip; ++i) dxs(i) = dx1(i) / 2.0f + dx1(i + 1) / 2.0f;
    for (int j = 0; j <= jp; ++j) dys(j) = dy1(j) / 2.0f + dy1(j + 1) / 2.0f;
    dzs(kp + 1) = dzs(kp);
    dzs(kp + 2) = dzs(kp + 1);
    dzs(-1) = dzs(0);
}

// grid.f95:22-82
void oracle_grid_reference(int ip, int jp, int kp, float *dx1_, float *dxl_, float *dy1_,
                           float *dyl_, float *z2_, float *dzn_, float *dzs_, float *dxs_,
                           float *dys_) {
    A1 dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1);
    for (int i = -1; i <= ip + 1; ++i) dx1(i) = 20.0f;
    for (int j = 0; j <= jp + 1; ++j) dy1(j) = 20.0f;
    dzn(0) = 2.5f;
    dzn(1) = 2.5f;
    for (int k = 2; k <= 15 && k <= kp + 2; ++k) dzn(k) = dzn(k - 1) * 1.05f;
    for (int k = 16; k <= 44 && k <= kp + 2; ++k) dzn(k) = 5.0f;
    for (int k = 45; k <= kp + 1; ++k) dzn(k) = dzn(k - 1) * 1.0459f;
    oracle_grid_metrics(ip, jp, kp, dx1_, dxl_, dy1_, dyl_, z2_, dzn_, dzs_, dxs_, dys_);
}

// feedbfm.f95:21-63 (zbm given instead of read from the GIS file).
void oracle_feedbfm(int km, int jm, int im, float *amask1_, float *bmask1_, float *cmask1_,
                    float *dmask1_, const float *zbm_, const float *z2_, const float *dzn_) {
    const int ip = im, jp = jm, kp = km;
    A3 amask1 = ARR_AM(amask1_), bmask1 = ARR_BM(bmask1_), cmask1 = ARR_CM(cmask1_),
       dmask1 = ARR_AM(dmask1_);
    A1 z2 = mk1(z2_, 1), dzn = mk1(dzn_, -1);
    const int zni = ip + 3;
    auto zbm = [&](int i, int j) { return zbm_[(size_t)(i + 1) + (size_t)zni * (size_t)(j + 1)]; };
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                amask1(i, j, k) = 1.0f;
                bmask1(i, j, k) = 0.0f;
                cmask1(i, j, k) = 0.0f;
                dmask1(i, j, k) = 0.0f;
            }
    for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i)
            for (int k = 1; k <= km; ++k)
                if (zbm(i, j) > z2(k) + 0.5f * dzn(k)) amask1(i, j, k) = 0.0f;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i)
                if (amask1(i, j, k) == 0.0f) {
                    bmask1(i, j, k) = 1.0f;
                    cmask1(i, j, k) = 1.0f;
                    dmask1(i, j, k) = 1.0f;
                }
}

// init.f95:46-107
void oracle_init(int km, int jm, int im, float *u_, float *v_, float *w_, float *p_, float *cn2s_,
                 const float *dxs_, float *cn2l_, float *cn3s_, const float *dys_, float *cn3l_,
                 const float *dzs_, float *cn4s_, float *cn4l_, float *cn1_, float *amask1,
                 float *bmask1, float *cmask1, float *dmask1, const float *zbm, const float *z2,
                 const float *dzn) {
    const int ip = im, jp = jm, kp = km;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_), p = ARR_P(p_), cn1 = ARR_I(cn1_);
    A1 dxs = mk1(dxs_, 0), dys = mk1(dys_, 0), dzs = mk1(dzs_, -1);
    A1 cn2s = mk1(cn2s_, 1), cn2l = mk1(cn2l_, 1), cn3s = mk1(cn3s_, 1), cn3l = mk1(cn3l_, 1),
       cn4s = mk1(cn4s_, 1), cn4l = mk1(cn4l_, 1);
    for (int k = 0; k <= kp + 1; ++k)
        for (int j = 0; j <= jp + 2; ++j)
            for (int i = 0; i <= ip + 2; ++i) p(i, j, k) = 0.0f;
    for (int k = 0; k <= kp + 1; ++k)
        for (int j = -1; j <= jp + 1; ++j)
            for (int i = 0; i <= ip + 1; ++i) {
                u(i, j, k) = 0.0f;
                v(i, j, k) = 0.0f;
            }
    for (int k = -1; k <= kp + 1; ++k)
        for (int j = -1; j <= jp + 1; ++j)
            for (int i = 0; i <= ip + 1; ++i) w(i, j, k) = 0.0f;
    oracle_feedbfm(km, jm, im, amask1, bmask1, cmask1, dmask1, zbm, z2, dzn);
    for (int i = 1; i <= im; ++i) {
        cn2s(i) = 2.0f / (dxs(i - 1) * (dxs(i - 1) + dxs(i)));
        cn2l(i) = 2.0f / (dxs(i) * (dxs(i - 1) + dxs(i)));
    }
    for (int j = 1; j <= jm; ++j) {
        cn3s(j) = 2.0f / (dys(j - 1) * (dys(j - 1) + dys(j)));
        cn3l(j) = 2.0f / (dys(j) * (dys(j - 1) + dys(j)));
    }
    for (int k = 1; k <= km; ++k) {
        const float dz1 = dzs(k - 1), dz2 = dzs(k);
        cn4s(k) = 2.0f / (dz1 * (dz1 + dz2));
        cn4l(k) = 2.0f / (dz2 * (dz1 + dz2));
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float c = 2.0f / (dxs(i - 1) * dxs(i)) + 2.0f / (dys(j - 1) * dys(j)) +
                          2.0f / (dz1 * dz2);
                cn1(i, j, k) = 1.0f / c;
            }
    }
}

// initial_wind_profile.f95:159-169 (bondv1_ext_wind_profile.f95 file)
void oracle_initial_wind_profile(float *wp_, int jm, int km, const float *z2_, const float *dzn_) {
    const int jp = jm;
    A1 z2 = mk1(z2_, 1), dzn = mk1(dzn_, -1);
    auto wp = [&](int j, int k) -> float & { return wp_[(size_t)(j - 1) + (size_t)jp * (k - 1)]; };
    for (int k = 1; k <= 78; ++k)
        for (int j = 1; j <= jm; ++j) wp(j, k) = 5.0f * std::pow((z2(k) + 0.5f * dzn(k)) / 600.0f, 0.2f);
    for (int k = 79; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) wp(j, k) = wp(j, 77);
}

// velnw.f95:27-59
void oracle_velnw(int km, int jm, int im, const float *p_, float ro, const float *dxs_, float *u_,
                  float dt, const float *f_, const float *dys_, float *v_, const float *g_,
                  const float *dzs_, float *w_, const float *h_) {
    const int ip = im, jp = jm, kp = km;
    A3 p = ARR_P(p_), u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_), f = ARR_F(f_), g = ARR_F(g_),
       h = ARR_F(h_);
    A1 dxs = mk1(dxs_, 0), dys = mk1(dys_, 0), dzs = mk1(dzs_, -1);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float pz = (-p(i, j, k) + p(i + 1, j, k)) / ro / dxs(i);
                u(i, j, k) = u(i, j, k) + dt * (f(i, j, k) - pz);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float pz = (-p(i, j, k) + p(i, j + 1, k)) / ro / dys(j);
                v(i, j, k) = v(i, j, k) + dt * (g(i, j, k) - pz);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float pz = (-p(i, j, k) + p(i, j, k + 1)) / ro / dzs(k);
                w(i, j, k) = w(i, j, k) + dt * (h(i, j, k) - pz);
            }
}

}  // extern "C"

namespace {

// bondv1.f95:67-137 / bondv1_ext_wind_profile.f95:57-127 (shared tail).
void bondv1_tail(int jm, float *u_, float *v_, float *w_, int km, int im, float dt,
                 const float *dxs_) {
    const int ip = im, jp = jm, kp = km;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    A1 dxs = mk1(dxs_, 0);
    float aaa = 0.0f, bbb = 0.0f;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
            const float x = u(im, j, k);
            aaa = (x > aaa) ? x : aaa;  // amax1
            bbb = (x < bbb) ? x : bbb;  // amin1
        }
    const float uout = (aaa + bbb) / 2.0f;
    g_last_uout = uout;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            u(im, j, k) = u(im, j, k) - dt * uout * (u(im, j, k) - u(im - 1, j, k)) / dxs(im);
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            v(im + 1, j, k) = v(im + 1, j, k) - dt * uout * (v(im + 1, j, k) - v(im, j, k)) / dxs(im);
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            w(im + 1, j, k) = w(im + 1, j, k) - dt * uout * (w(im + 1, j, k) - w(im, j, k)) / dxs(im);
    // side flow condition; periodic
    for (int k = 0; k <= km + 1; ++k)
        for (int i = 0; i <= im + 1; ++i) {
            u(i, 0, k) = u(i, jm, k);
            u(i, jm + 1, k) = u(i, 1, k);
        }
    for (int k = 0; k <= km + 1; ++k)
        for (int i = 0; i <= im + 1; ++i) {
            v(i, 0, k) = v(i, jm, k);
            v(i, jm + 1, k) = v(i, 1, k);
        }
    for (int k = 0; k <= km; ++k)
        for (int i = 0; i <= im + 1; ++i) {
            w(i, 0, k) = w(i, jm, k);
            w(i, jm + 1, k) = w(i, 1, k);
        }
    // top and underground condition
    for (int j = 0; j <= jm + 1; ++j)
        for (int i = 0; i <= im + 1; ++i) {
            u(i, j, 0) = -u(i, j, 1);
            u(i, j, km + 1) = u(i, j, km);
        }
    for (int j = 0; j <= jm + 1; ++j)
        for (int i = 0; i <= im + 1; ++i) {
            v(i, j, 0) = -v(i, j, 1);
            v(i, j, km + 1) = v(i, j, km);
        }
    // bondv1.f95:132-137 runs i from -1, one below w's lower bound 0.  In the
    // column-major layout w(-1,j,k) is the element w(ip+1,j-1,k) (for j=-1:
    // w(ip+1,jp+1,k-1)).  Restated with that aliasing made explicit.
    for (int j = -1; j <= jm + 1; ++j)
        for (int i = -1; i <= im + 1; ++i) {
            if (i == -1) {
                if (j >= 0) {
                    w(ip + 1, j - 1, 0) = 0.0f;
                    w(ip + 1, j - 1, km) = 0.0f;
                } else {
                    w(ip + 1, jp + 1, -1) = 0.0f;
                    w(ip + 1, jp + 1, km - 1) = 0.0f;
                }
            } else {
                w(i, j, 0) = 0.0f;
                w(i, j, km) = 0.0f;
            }
        }
}

// bondv1.f95:47-59 (ICAL=0): n==1 broadcast of the i=1 inflow plane.
void bondv1_n1(float *u_, float *v_, float *w_, int im, int jm, int km, int n) {
    const int ip = im, jp = jm, kp = km;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    if (n != 1) return;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 2; i <= im; ++i) {
                u(i, j, k) = u(1, j, k);
                v(i, j, k) = v(1, j, k);
                w(i, j, k) = w(1, j, k);
            }
}

}  // namespace

extern "C" {

// bondv1.f95:26-137
void oracle_bondv1(int jm, float *u_, const float *z2_, const float *dzn_, float *v_, float *w_,
                   int km, int n, int im, float dt, const float *dxs) {
    const int ip = im, jp = jm, kp = km;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    A1 z2 = mk1(z2_, 1), dzn = mk1(dzn_, -1);
    for (int i = 0; i <= 1; ++i)
        for (int k = 1; k <= 78; ++k)
            for (int j = 1; j <= jm; ++j) {
                const float u_val = 5.0f * std::pow((z2(k) + 0.5f * dzn(k)) / 600.0f, 0.2f);
                u(i, j, k) = u_val;
                v(i, j, k) = 0.0f;
                w(i, j, k) = 0.0f;
            }
    for (int i = 0; i <= 1; ++i)
        for (int k = 79; k <= km; ++k)
            for (int j = 1; j <= jm; ++j) {
                u(i, j, k) = u(i, j, 77);
                v(i, j, k) = 0.0f;
                w(i, j, k) = 0.0f;
            }
    bondv1_n1(u_, v_, w_, im, jm, km, n);
    bondv1_tail(jm, u_, v_, w_, km, im, dt, dxs);
}

// bondv1_ext_wind_profile.f95:27-127
void oracle_bondv1_ext_wind_profile(int jm, float *u_, const float *z2, const float *dzn, float *v_,
                                    float *w_, int km, int n, int im, float dt, const float *dxs,
                                    const float *wp_) {
    const int ip = im, jp = jm, kp = km;
    (void)z2;
    (void)dzn;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    auto wp = [&](int j, int k) { return wp_[(size_t)(j - 1) + (size_t)jp * (k - 1)]; };
    for (int i = 0; i <= 1; ++i)
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j) {
                u(i, j, k) = wp(j, k);
                v(i, j, k) = 0.0f;
                w(i, j, k) = 0.0f;
            }
    bondv1_n1(u_, v_, w_, im, jm, km, n);
    bondv1_tail(jm, u_, v_, w_, km, im, dt, dxs);
}

// vel2.f95:48-188
void oracle_vel2(int km, int jm, int im, float *nou1_, const float *u_, float *diu1_,
                 const float *dx1_, float *nou5_, const float *v_, float *diu5_, const float *dy1_,
                 float *nou9_, const float *w_, float *diu9_, const float *dzn_, float *cov1_,
                 float *cov5_, float *cov9_, float *nou2_, float *diu2_, float *cov2_, float *nou3_,
                 float *diu3_, const float *dzs_, float *cov3_, float *nou4_, float *diu4_,
                 float *cov4_, float *nou6_, float *diu6_, float *cov6_, float *nou7_, float *diu7_,
                 float *cov7_, float *nou8_, float *diu8_, float *cov8_) {
    const int ip = im, jp = jm, kp = km;
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    A3 nou1 = ARR_D15(nou1_), diu1 = ARR_D15(diu1_), cov1 = ARR_D15(cov1_);
    A3 nou5 = ARR_D15(nou5_), diu5 = ARR_D15(diu5_), cov5 = ARR_D15(cov5_);
    A3 nou2 = ARR_D(nou2_), diu2 = ARR_D(diu2_), cov2 = ARR_D(cov2_);
    A3 nou3 = ARR_D(nou3_), diu3 = ARR_D(diu3_), cov3 = ARR_D(cov3_);
    A3 nou4 = ARR_D(nou4_), diu4 = ARR_D(diu4_), cov4 = ARR_D(cov4_);
    A3 nou6 = ARR_D(nou6_), diu6 = ARR_D(diu6_), cov6 = ARR_D(cov6_);
    A3 nou7 = ARR_D(nou7_), diu7 = ARR_D(diu7_), cov7 = ARR_D(cov7_);
    A3 nou8 = ARR_D(nou8_), diu8 = ARR_D(diu8_), cov8 = ARR_D(cov8_);
    A3 nou9 = ARR_D(nou9_), diu9 = ARR_D(diu9_), cov9 = ARR_D(cov9_);
    A1 dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1), dzs = mk1(dzs_, -1);
    const float u0 = 0.0f;  // integer parameter u0 = 0 (vel2.f95:46)
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou1(i, j, k) = (u(i - 1, j, k) + u(i, j, k)) / 2.0f;
                diu1(i, j, k) = (-u(i - 1, j, k) + u(i, j, k)) / dx1(i);
                nou5(i, j, k) = (v(i, j - 1, k) + v(i, j, k)) / 2.0f;
                diu5(i, j, k) = (-v(i, j - 1, k) + v(i, j, k)) / dy1(j);
                nou9(i, j, k) = (w(i, j, k - 1) + w(i, j, k)) / 2.0f;
                diu9(i, j, k) = (-w(i, j, k - 1) + w(i, j, k)) / dzn(k);
                cov1(i, j, k) = nou1(i, j, k) * diu1(i, j, k);
                cov5(i, j, k) = nou5(i, j, k) * diu5(i, j, k);
                cov9(i, j, k) = nou9(i, j, k) * diu9(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou2(i, j, k) = (dx1(i + 1) * v(i, j - 1, k) + dx1(i) * v(i + 1, j - 1, k)) /
                                (dx1(i) + dx1(i + 1));
                diu2(i, j, k) = 2.0f * (-u(i, j - 1, k) + u(i, j, k)) / (dy1(j - 1) + dy1(j));
                cov2(i, j, k) = nou2(i, j, k) * diu2(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km + 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou3(i, j, k) = (dx1(i + 1) * w(i, j, k - 1) + dx1(i) * w(i + 1, j, k - 1)) /
                                (dx1(i) + dx1(i + 1));
                diu3(i, j, k) = (-u(i, j, k - 1) + u(i, j, k)) / dzs(k - 1);
                cov3(i, j, k) = nou3(i, j, k) * diu3(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou4(i, j, k) = (dy1(j + 1) * u(i - 1, j, k) + dy1(j) * u(i - 1, j + 1, k)) /
                                (dy1(j) + dy1(j + 1));
                diu4(i, j, k) = 2.0f * (-v(i - 1, j, k) + v(i, j, k)) / (dx1(i - 1) + dx1(i));
                cov4(i, j, k) = (nou4(i, j, k) - u0) * diu4(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km + 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou6(i, j, k) = (dy1(j + 1) * w(i, j, k - 1) + dy1(j) * w(i, j + 1, k - 1)) /
                                (dy1(j) + dy1(j + 1));
                diu6(i, j, k) = (-v(i, j, k - 1) + v(i, j, k)) / dzs(k - 1);
                cov6(i, j, k) = nou6(i, j, k) * diu6(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou7(i, j, k) = (dzn(k + 1) * u(i - 1, j, k) + dzn(k) * u(i - 1, j, k + 1)) /
                                (dzn(k) + dzn(k + 1));
                diu7(i, j, k) = 2.0f * (-w(i - 1, j, k) + w(i, j, k)) / (dx1(i - 1) + dx1(i));
                cov7(i, j, k) = (nou7(i, j, k) - u0) * diu7(i, j, k);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                nou8(i, j, k) = (dzn(k + 1) * v(i, j - 1, k) + dzn(k) * v(i, j - 1, k + 1)) /
                                (dzn(k) + dzn(k + 1));
                diu8(i, j, k) = 2.0f * (-w(i, j - 1, k) + w(i, j, k)) / (dy1(j - 1) + dy1(j));
                cov8(i, j, k) = nou8(i, j, k) * diu8(i, j, k);
            }
    // boundary copies, vel2.f95:125-188
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
            nou1(im + 1, j, k) = nou1(im, j, k);
            diu1(im + 1, j, k) = diu1(im, j, k);
            cov1(im + 1, j, k) = cov1(im, j, k);
        }
    for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
            nou2(i, 0, k) = nou2(i, jm, k);
            diu2(i, 0, k) = diu2(i, jm, k);
            cov2(i, 0, k) = cov2(i, jm, k);
            nou2(i, jm + 1, k) = nou2(i, 1, k);
            diu2(i, jm + 1, k) = diu2(i, 1, k);
            cov2(i, jm + 1, k) = cov2(i, 1, k);
        }
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
            nou4(im + 1, j, k) = nou4(im, j, k);
            diu4(im + 1, j, k) = diu4(im, j, k);
            cov4(im + 1, j, k) = cov4(im, j, k);
        }
    for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
            nou5(i, 0, k) = nou5(i, jm, k);
            diu5(i, 0, k) = diu5(i, jm, k);
            cov5(i, 0, k) = cov5(i, jm, k);
            nou5(i, jm + 1, k) = nou5(i, 1, k);
            diu5(i, jm + 1, k) = diu5(i, 1, k);
            cov5(i, jm + 1, k) = cov5(i, 1, k);
        }
    for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm; ++j) {
            nou7(im + 1, j, k) = nou7(im, j, k);
            diu7(im + 1, j, k) = diu7(im, j, k);
            cov7(im + 1, j, k) = cov7(im, j, k);
        }
    for (int k = 1; k <= km - 1; ++k)
        for (int i = 1; i <= im; ++i) {
            nou8(i, 0, k) = nou8(i, jm, k);
            diu8(i, 0, k) = diu8(i, jm, k);
            cov8(i, 0, k) = cov8(i, jm, k);
            nou8(i, jm + 1, k) = nou8(i, 1, k);
            diu8(i, jm + 1, k) = diu8(i, 1, k);
            cov8(i, jm + 1, k) = cov8(i, 1, k);
        }
    for (int k = 1; k <= km + 1; ++k)
        for (int j = 1; j <= jm + 1; ++j) {
            diu2(im + 1, j, k) = diu2(im, j, k);
            diu3(im + 1, j, k) = diu3(im, j, k);
        }
    for (int k = 1; k <= km + 1; ++k)
        for (int i = 1; i <= im + 1; ++i) {
            diu4(i, 0, k) = diu4(i, jm, k);
            diu6(i, 0, k) = diu6(i, jm, k);
        }
}

// velFG.f95:56-105
void oracle_velfg(int km, int jm, int im, const float *dx1_, float *cov1_, float *cov2_,
                  float *cov3_, float *dfu1_, float *diu1_, float *diu2_, const float *dy1_,
                  float *diu3_, const float *dzn_, float vn, float *f_, float *cov4_, float *cov5_,
                  float *cov6_, float *dfv1_, float *diu4_, float *diu5_, float *diu6_, float *g_,
                  float *cov7_, float *cov8_, float *cov9_, float *dfw1_, float *diu7_,
                  float *diu8_, float *diu9_, const float *dzs_, float *h_, float *nou1,
                  const float *u, float *nou5, const float *v, float *nou9, const float *w,
                  float *nou2, float *nou3, float *nou4, float *nou6, float *nou7, float *nou8) {
    const int ip = im, jp = jm, kp = km;
    oracle_vel2(km, jm, im, nou1, u, diu1_, dx1_, nou5, v, diu5_, dy1_, nou9, w, diu9_, dzn_, cov1_,
                cov5_, cov9_, nou2, diu2_, cov2_, nou3, diu3_, dzs_, cov3_, nou4, diu4_, cov4_, nou6,
                diu6_, cov6_, nou7, diu7_, cov7_, nou8, diu8_, cov8_);
    A3 cov1 = ARR_D15(cov1_), cov5 = ARR_D15(cov5_), diu1 = ARR_D15(diu1_), diu5 = ARR_D15(diu5_);
    A3 cov2 = ARR_D(cov2_), cov3 = ARR_D(cov3_), cov4 = ARR_D(cov4_), cov6 = ARR_D(cov6_),
       cov7 = ARR_D(cov7_), cov8 = ARR_D(cov8_), cov9 = ARR_D(cov9_);
    A3 diu2 = ARR_D(diu2_), diu3 = ARR_D(diu3_), diu4 = ARR_D(diu4_), diu6 = ARR_D(diu6_),
       diu7 = ARR_D(diu7_), diu8 = ARR_D(diu8_), diu9 = ARR_D(diu9_);
    A3 dfu1 = ARR_DFU(dfu1_), dfv1 = ARR_DFV(dfv1_), dfw1 = ARR_I(dfw1_);
    A3 f = ARR_F(f_), g = ARR_F(g_), h = ARR_F(h_);
    A1 dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1), dzs = mk1(dzs_, -1);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float covx1 = (dx1(i + 1) * cov1(i, j, k) + dx1(i) * cov1(i + 1, j, k)) /
                              (dx1(i) + dx1(i + 1));
                float covy1 = (cov2(i, j, k) + cov2(i, j + 1, k)) / 2.0f;
                float covz1 = (cov3(i, j, k) + cov3(i, j, k + 1)) / 2.0f;
                float covc = covx1 + covy1 + covz1;
                dfu1(i, j, k) = 2.0f * (-diu1(i, j, k) + diu1(i + 1, j, k)) / (dx1(i) + dx1(i + 1)) +
                                (-diu2(i, j, k) + diu2(i, j + 1, k)) / dy1(j) +
                                (-diu3(i, j, k) + diu3(i, j, k + 1)) / dzn(k);
                float df = vn * dfu1(i, j, k);
                f(i, j, k) = (-covc + df);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float covx1 = (cov4(i, j, k) + cov4(i + 1, j, k)) / 2.0f;
                float covy1 = (dy1(j + 1) * cov5(i, j, k) + dy1(j) * cov5(i, j + 1, k)) /
                              (dy1(j) + dy1(j + 1));
                float covz1 = (cov6(i, j, k) + cov6(i, j, k + 1)) / 2.0f;
                float covc = covx1 + covy1 + covz1;
                dfv1(i, j, k) = (-diu4(i, j, k) + diu4(i + 1, j, k)) / dx1(i) +
                                2.0f * (-diu5(i, j, k) + diu5(i, j + 1, k)) / (dy1(j) + dy1(j + 1)) +
                                (-diu6(i, j, k) + diu6(i, j, k + 1)) / dzn(k);
                float df = vn * dfv1(i, j, k);
                g(i, j, k) = (-covc + df);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float covx1 = (cov7(i, j, k) + cov7(i + 1, j, k)) / 2.0f;
                float covy1 = (cov8(i, j, k) + cov8(i, j + 1, k)) / 2.0f;
                float covz1 = (dzn(k + 1) * cov9(i, j, k) + dzn(k) * cov9(i, j, k + 1)) /
                              (dzn(k) + dzn(k + 1));
                float covc = covx1 + covy1 + covz1;
                dfw1(i, j, k) = (-diu7(i, j, k) + diu7(i + 1, j, k)) / dx1(i) +
                                (-diu8(i, j, k) + diu8(i, j + 1, k)) / dy1(j) +
                                (-diu9(i, j, k) + diu9(i, j, k + 1)) / dzs(k);
                float df = vn * dfw1(i, j, k);
                h(i, j, k) = (-covc + df);
            }
}

// feedbf.f95:38-67
void oracle_feedbf(int km, int jm, int im, float *usum_, const float *u_, const float *bmask1_,
                   float *vsum_, const float *v_, const float *cmask1_, float *wsum_,
                   const float *w_, const float *dmask1_, float alpha, float dt, float beta,
                   float *fx_, float *fy_, float *fz_, float *f_, float *g_, float *h_) {
    const int ip = im, jp = jm, kp = km;
    A3 usum = ARR_F(usum_), vsum = ARR_F(vsum_), wsum = ARR_F(wsum_), fx = ARR_F(fx_),
       fy = ARR_F(fy_), fz = ARR_F(fz_), f = ARR_F(f_), g = ARR_F(g_), h = ARR_F(h_);
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_);
    A3 bmask1 = ARR_BM(bmask1_), cmask1 = ARR_CM(cmask1_), dmask1 = ARR_AM(dmask1_);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                usum(i, j, k) = (usum(i, j, k) + u(i, j, k)) * bmask1(i, j, k);
                vsum(i, j, k) = (vsum(i, j, k) + v(i, j, k)) * cmask1(i, j, k);
                wsum(i, j, k) = (wsum(i, j, k) + w(i, j, k)) * dmask1(i, j, k);
                float f1x = alpha * usum(i, j, k) * dt;
                float f1y = alpha * vsum(i, j, k) * dt;
                float f1z = alpha * wsum(i, j, k) * dt;
                float f2x = beta * u(i, j, k) * bmask1(i, j, k);
                float f2y = beta * v(i, j, k) * cmask1(i, j, k);
                float f2z = beta * w(i, j, k) * dmask1(i, j, k);
                fx(i, j, k) = f1x + f2x;
                fy(i, j, k) = f1y + f2y;
                fz(i, j, k) = f1z + f2z;
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                f(i, j, k) = f(i, j, k) + fx(i, j, k);
                g(i, j, k) = g(i, j, k) + fy(i, j, k);
                h(i, j, k) = h(i, j, k) + fz(i, j, k);
            }
}

// boundsm.f95:13-32
void oracle_boundsm(int km, int jm, float *sm_, int im) {
    const int ip = im, jp = jm, kp = km;
    A3 sm = ARR_SM(sm_);
    for (int k = 0; k <= km + 1; ++k)
        for (int j = -1; j <= jm + 1; ++j) {
            sm(0, j, k) = sm(1, j, k);
            sm(im + 1, j, k) = sm(im, j, k);
        }
    for (int k = 0; k <= km + 1; ++k)
        for (int i = 0; i <= im + 1; ++i) {
            sm(i, jm + 1, k) = sm(i, jm, k);
            sm(i, 0, k) = sm(i, 1, k);
        }
    for (int j = -1; j <= jm + 1; ++j)
        for (int i = 0; i <= im + 1; ++i) {
            sm(i, j, 0) = -sm(i, j, 1);
            sm(i, j, km + 1) = sm(i, j, km);
        }
}

// les.f95:31-182
void oracle_les(int km, float *delx1_, const float *dx1_, const float *dy1_, const float *dzn_,
                int jm, int im, const float *diu1_, const float *diu2_, const float *diu3_,
                const float *diu4_, const float *diu5_, const float *diu6_, const float *diu7_,
                const float *diu8_, const float *diu9_, float *sm_, float *f_, float *g_,
                float *h_) {
    const int ip = im, jp = jm, kp = km;
    A3 diu1 = ARR_D15(diu1_), diu5 = ARR_D15(diu5_);
    A3 diu2 = ARR_D(diu2_), diu3 = ARR_D(diu3_), diu4 = ARR_D(diu4_), diu6 = ARR_D(diu6_),
       diu7 = ARR_D(diu7_), diu8 = ARR_D(diu8_), diu9 = ARR_D(diu9_);
    A3 sm = ARR_SM(sm_), f = ARR_F(f_), g = ARR_F(g_), h = ARR_F(h_);
    A1 delx1 = mk1(delx1_, 1), dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1);
    const float cs0 = 0.1f;
    for (int k = 1; k <= km; ++k) delx1(k) = std::pow(dx1(0) * dy1(0) * dzn(k), 1.0f / 3.0f);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float dudxx1 = diu1(i, j, k);
                float dudyx1 = (diu2(i - 1, j, k) + diu2(i - 1, j + 1, k) + diu2(i, j, k) +
                                diu2(i, j + 1, k)) * 0.25f;
                float dudzx1 = (diu3(i - 1, j, k) + diu3(i - 1, j, k + 1) + diu3(i, j, k) +
                                diu3(i, j, k + 1)) * 0.25f;
                float dvdxx1 = (diu4(i, j, k) + diu4(i, j - 1, k) + diu4(i + 1, j, k) +
                                diu4(i + 1, j - 1, k)) * 0.25f;
                float dvdyx1 = diu5(i, j, k);
                float dvdzx1 = (diu6(i, j - 1, k) + diu6(i, j - 1, k + 1) + diu6(i, j, k) +
                                diu6(i, j, k + 1)) * 0.25f;
                float dwdxx1 = (diu7(i, j, k) + diu7(i, j, k - 1) + diu7(i + 1, j, k) +
                                diu7(i + 1, j, k - 1)) * 0.25f;
                float dwdyx1 = (diu8(i, j, k) + diu8(i, j, k - 1) + diu8(i, j + 1, k) +
                                diu8(i, j + 1, k - 1)) * 0.25f;
                float dwdzx1 = diu9(i, j, k);
                float csx1 = cs0;
                float cd = csx1 * delx1(k);
                float a = dudyx1 + dvdxx1, b = dwdyx1 + dvdzx1, c = dudzx1 + dwdxx1;
                sm(i, j, k) = (cd * cd) *
                              std::sqrt(2.0f * (dudxx1 * dudxx1 + dvdyx1 * dvdyx1 + dwdzx1 * dwdzx1) +
                                        a * a + b * b + c * c);
            }
    oracle_boundsm(km, jm, sm_, im);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float evsx2 = sm(i + 1, j, k);
                float evsx1 = sm(i, j, k);
                float evsy2 = (dy1(j + 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dy1(j) * ((dx1(i + 1) * sm(i, j + 1, k) + dx1(i) * sm(i + 1, j + 1, k)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dy1(j) + dy1(j + 1));
                float evsy1 = (dy1(j + 1) * ((dx1(i + 1) * sm(i, j - 1, k) + dx1(i) * sm(i + 1, j - 1, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dy1(j) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dy1(j) + dy1(j + 1));
                float evsz2 = (dzn(k + 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dzn(k) * ((dx1(i + 1) * sm(i, j, k + 1) + dx1(i) * sm(i + 1, j, k + 1)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dzn(k) + dzn(k + 1));
                float evsz1 = (dzn(k) * ((dx1(i + 1) * sm(i, j, k - 1) + dx1(i) * sm(i + 1, j, k - 1)) /
                                         (dx1(i) + dx1(i + 1))) +
                               dzn(k - 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1)))) /
                              (dzn(k - 1) + dzn(k));
                float visux2 = (evsx2) * 2.0f * diu1(i + 1, j, k);
                float visux1 = (evsx1) * 2.0f * diu1(i, j, k);
                float visuy2 = (evsy2) * (diu2(i, j + 1, k) + diu4(i + 1, j, k));
                float visuy1 = (evsy1) * (diu2(i, j, k) + diu4(i + 1, j - 1, k));
                float visuz2 = (evsz2) * (diu3(i, j, k + 1) + diu7(i + 1, j, k));
                float visuz1 = (evsz1) * (diu3(i, j, k) + diu7(i + 1, j, k - 1));
                float vfu = (visux2 - visux1) / dx1(i) + (visuy2 - visuy1) / dy1(j) +
                            (visuz2 - visuz1) / dzn(k);
                f(i, j, k) = (f(i, j, k) + vfu);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float evsy2 = sm(i, j + 1, k);
                float evsy1 = sm(i, j, k);
                float evsx2 = (dy1(j + 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dy1(j) * ((dx1(i + 1) * sm(i, j + 1, k) + dx1(i) * sm(i + 1, j + 1, k)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dy1(j) + dy1(j + 1));
                float evsx1 = (dy1(j + 1) * ((dx1(i) * sm(i - 1, j, k) + dx1(i - 1) * sm(i, j, k)) /
                                             (dx1(i - 1) + dx1(i))) +
                               dy1(j) * ((dx1(i) * sm(i - 1, j + 1, k) + dx1(i - 1) * sm(i, j + 1, k)) /
                                         (dx1(i - 1) + dx1(i)))) /
                              (dy1(j) + dy1(j + 1));
                float evsz2 = (dzn(k + 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dzn(k) * ((dx1(i + 1) * sm(i, j, k + 1) + dx1(i) * sm(i + 1, j, k + 1)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dzn(k) + dzn(k + 1));
                float evsz1 = (dzn(k) * ((dx1(i + 1) * sm(i, j, k - 1) + dx1(i) * sm(i + 1, j, k - 1)) /
                                         (dx1(i) + dx1(i + 1))) +
                               dzn(k - 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1)))) /
                              (dzn(k - 1) + dzn(k));
                float visvx2 = (evsx2) * (diu2(i, j + 1, k) + diu4(i + 1, j, k));
                float visvx1 = (evsx1) * (diu2(i - 1, j + 1, k) + diu4(i, j, k));
                float visvy2 = (evsy2) * 2.0f * diu5(i, j + 1, k);
                float visvy1 = (evsy1) * 2.0f * diu5(i, j, k);
                float visvz2 = (evsz2) * (diu6(i, j, k + 1) + diu8(i, j + 1, k));
                float visvz1 = (evsz1) * (diu6(i, j, k) + diu8(i, j + 1, k - 1));
                float vfv = (visvx2 - visvx1) / dx1(i) + (visvy2 - visvy1) / dy1(j) +
                            (visvz2 - visvz1) / dzn(k);
                g(i, j, k) = (g(i, j, k) + vfv);
            }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float evsz2 = sm(i, j, k + 1);
                float evsz1 = sm(i, j, k);
                float evsx2 = (dzn(k + 1) * ((dx1(i + 1) * sm(i, j, k) + dx1(i) * sm(i + 1, j, k)) /
                                             (dx1(i) + dx1(i + 1))) +
                               dzn(k) * ((dx1(i + 1) * sm(i, j, k + 1) + dx1(i) * sm(i + 1, j, k + 1)) /
                                         (dx1(i) + dx1(i + 1)))) /
                              (dzn(k) + dzn(k + 1));
                float evsx1 = (dzn(k + 1) * ((dx1(i) * sm(i - 1, j, k) + dx1(i - 1) * sm(i, j, k)) /
                                             (dx1(i - 1) + dx1(i))) +
                               dzn(k) * ((dx1(i) * sm(i - 1, j, k + 1) + dx1(i - 1) * sm(i, j, k + 1)) /
                                         (dx1(i - 1) + dx1(i)))) /
                              (dzn(k) + dzn(k + 1));
                float evsy2 = (dzn(k + 1) * ((dy1(j + 1) * sm(i, j, k) + dy1(j) * sm(i, j + 1, k)) /
                                             (dy1(j) + dy1(j + 1))) +
                               dzn(k) * ((dy1(j + 1) * sm(i, j, k + 1) + dy1(j) * sm(i, j + 1, k + 1)) /
                                         (dy1(j) + dy1(j + 1)))) /
                              (dzn(k) + dzn(k + 1));
                float evsy1 = (dzn(k + 1) * ((dy1(j) * sm(i, j - 1, k) + dy1(j - 1) * sm(i, j, k)) /
                                             (dy1(j - 1) + dy1(j))) +
                               dzn(k) * ((dy1(j) * sm(i, j - 1, k + 1) + dy1(j - 1) * sm(i, j, k + 1)) /
                                         (dy1(j - 1) + dy1(j)))) /
                              (dzn(k) + dzn(k + 1));
                float viswx2 = (evsx2) * (diu3(i, j, k + 1) + diu7(i + 1, j, k));
                float viswx1 = (evsx1) * (diu3(i - 1, j, k + 1) + diu7(i, j, k));
                float viswy2 = (evsy2) * (diu6(i, j, k + 1) + diu8(i, j + 1, k));
                float viswy1 = (evsy1) * (diu6(i, j - 1, k + 1) + diu8(i, j, k));
                float viswz2 = (evsz2) * 2.0f * diu9(i, j, k + 1);
                float viswz1 = (evsz1) * 2.0f * diu9(i, j, k);
                float vfw = (viswx2 - viswx1) / dx1(i) + (viswy2 - viswy1) / dy1(j) +
                            (viswz2 - viswz1) / dzn(k);
                h(i, j, k) = (h(i, j, k) + vfw);
            }
}

// adam.f95:32-46 (the data21 file write at n%1000==0 is omitted)
void oracle_adam(int n, int nmax, float *fold_, int im, int jm, int km, float *gold_,
                 float *hold_, float *f_, float *g_, float *h_) {
    (void)n;
    (void)nmax;
    const int ip = im, jp = jm, kp = km;
    A3 fold = ARR_I(fold_), gold = ARR_I(gold_), hold = ARR_I(hold_);
    A3 f = ARR_F(f_), g = ARR_F(g_), h = ARR_F(h_);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                float fd = f(i, j, k), gd = g(i, j, k), hd = h(i, j, k);
                f(i, j, k) = 1.5f * f(i, j, k) - 0.5f * fold(i, j, k);
                g(i, j, k) = 1.5f * g(i, j, k) - 0.5f * gold(i, j, k);
                h(i, j, k) = 1.5f * h(i, j, k) - 0.5f * hold(i, j, k);
                fold(i, j, k) = fd;
                gold(i, j, k) = gd;
                hold(i, j, k) = hd;
            }
}

// aveflow.f95:42-157 (the data10/data11 writes of :159-174 are left to the
// caller).  Serial loops in the Fortran order.  At k = 1 the finish of uwfx
// (:112-113) reads aveu(i,j,0), avew(i,j,0) and avew(i+1,j,0): they are
// taken at their flattened index in the (ip,jp,kp) arrays, 0 where that
// index lies before the first element (outside the arrays in the reference).
void oracle_aveflow(int n, int n1, int km, int jm, int im, float *aveu_, float *avev_, float *avew_,
                    float *avep_, float *avel_, float *aveuu_, float *avevv_, float *aveww_,
                    float *avesm_, float *avesmsm_, float *uwfx_, float *avesu_, float *avesv_,
                    float *avesw_, float *avesuu_, float *avesvv_, float *avesww_, const float *u_,
                    const float *v_, const float *w_, const float *p_, const float *sm_, int nmax,
                    float *uwfxs_) {
    const int ip = im, jp = jm, kp = km;
    A3 aveu = ARR_I(aveu_), avev = ARR_I(avev_), avew = ARR_I(avew_), avep = ARR_I(avep_);
    A3 avel = ARR_I(avel_), aveuu = ARR_I(aveuu_), avevv = ARR_I(avevv_), aveww = ARR_I(aveww_);
    A3 avesm = ARR_I(avesm_), avesmsm = ARR_I(avesmsm_), uwfx = ARR_I(uwfx_);
    A3 avesu = mk(avesu_, 1, ip, 1, kp, 1, 1), avesv = mk(avesv_, 1, ip, 1, kp, 1, 1);
    A3 avesw = mk(avesw_, 1, ip, 1, kp, 1, 1), avesuu = mk(avesuu_, 1, ip, 1, kp, 1, 1);
    A3 avesvv = mk(avesvv_, 1, ip, 1, kp, 1, 1), avesww = mk(avesww_, 1, ip, 1, kp, 1, 1);
    A3 uwfxs = mk(uwfxs_, 1, ip, 1, kp, 1, 1);
    A3 u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_), p = ARR_P(p_), sm = ARR_SM(sm_);
    // the flattened read of the uwfx finish
    auto flat = [&](const float *a, int i, int j, int k) {
        const long long idx = (long long)(i - 1) + (long long)ip * ((j - 1) + (long long)jp * (k - 1));
        return idx < 0 ? 0.0f : a[idx];
    };
    if (n == n1) {
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    aveu(i, j, k) = 0.0f;
                    avev(i, j, k) = 0.0f;
                    avew(i, j, k) = 0.0f;
                    avep(i, j, k) = 0.0f;
                    avel(i, j, k) = 0.0f;
                    aveuu(i, j, k) = 0.0f;
                    avevv(i, j, k) = 0.0f;
                    aveww(i, j, k) = 0.0f;
                    avesm(i, j, k) = 0.0f;
                    avesmsm(i, j, k) = 0.0f;
                    uwfx(i, j, k) = 0.0f;
                }
        for (int k = 1; k <= km; ++k)
            for (int i = 1; i <= im; ++i) {
                avesu(i, k, 1) = 0.0f;
                avesv(i, k, 1) = 0.0f;
                avesw(i, k, 1) = 0.0f;
                avesuu(i, k, 1) = 0.0f;
                avesvv(i, k, 1) = 0.0f;
                avesww(i, k, 1) = 0.0f;
            }
    }
    if (n >= n1) {
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    aveu(i, j, k) = aveu(i, j, k) + u(i, j, k);
                    avev(i, j, k) = avev(i, j, k) + v(i, j, k);
                    avew(i, j, k) = avew(i, j, k) + w(i, j, k);
                    avep(i, j, k) = avep(i, j, k) + p(i, j, k);
                    aveuu(i, j, k) = aveuu(i, j, k) + u(i, j, k) * u(i, j, k);
                    avevv(i, j, k) = avevv(i, j, k) + v(i, j, k) * v(i, j, k);
                    aveww(i, j, k) = aveww(i, j, k) + w(i, j, k) * w(i, j, k);
                    avesm(i, j, k) = avesm(i, j, k) + sm(i, j, k);
                    avesmsm(i, j, k) = avesmsm(i, j, k) + sm(i, j, k) * sm(i, j, k);
                    uwfx(i, j, k) = uwfx(i, j, k) + 0.5f * (u(i, j, k - 1) + u(i, j, k)) * 0.5f *
                                                        (w(i, j, k - 1) + w(i + 1, j, k - 1));
                }
    }
    if (n == nmax) {
        const float cnt = (float)(nmax - n1 + 1);
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    aveu(i, j, k) = aveu(i, j, k) / cnt;
                    avev(i, j, k) = avev(i, j, k) / cnt;
                    avew(i, j, k) = avew(i, j, k) / cnt;
                    avep(i, j, k) = avep(i, j, k) / cnt;
                    avel(i, j, k) = avel(i, j, k) / cnt;
                    aveuu(i, j, k) = aveuu(i, j, k) / cnt;
                    avevv(i, j, k) = avevv(i, j, k) / cnt;
                    aveww(i, j, k) = aveww(i, j, k) / cnt;
                    avesm(i, j, k) = avesm(i, j, k) / cnt;
                    avesmsm(i, j, k) = avesmsm(i, j, k) / cnt;
                }
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i)
                    uwfx(i, j, k) = uwfx(i, j, k) / cnt - 0.5f * (flat(aveu_, i, j, k - 1) + aveu(i, j, k)) * 0.5f *
                                                              (flat(avew_, i, j, k - 1) + flat(avew_, i + 1, j, k - 1));
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    avesu(i, k, 1) = avesu(i, k, 1) + aveu(i, j, k);
                    avesv(i, k, 1) = avesv(i, k, 1) + avev(i, j, k);
                    avesw(i, k, 1) = avesw(i, k, 1) + avew(i, j, k);
                    avesuu(i, k, 1) = avesuu(i, k, 1) + aveuu(i, j, k);
                    avesvv(i, k, 1) = avesvv(i, k, 1) + avevv(i, j, k);
                    avesww(i, k, 1) = avesww(i, k, 1) + aveww(i, j, k);
                    uwfxs(i, k, 1) = uwfxs(i, k, 1) + uwfx(i, j, k);
                }
        const float rjm = (float)jm;
        for (int k = 1; k <= km; ++k)
            for (int i = 1; i <= im; ++i) {
                avesu(i, k, 1) = avesu(i, k, 1) / rjm;
                avesv(i, k, 1) = avesv(i, k, 1) / rjm;
                avesw(i, k, 1) = avesw(i, k, 1) / rjm;
                avesuu(i, k, 1) = avesuu(i, k, 1) / rjm;
                avesvv(i, k, 1) = avesvv(i, k, 1) / rjm;
                avesww(i, k, 1) = avesww(i, k, 1) / rjm;
                uwfxs(i, k, 1) = uwfxs(i, k, 1) / rjm;
            }
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    aveuu(i, j, k) = std::sqrt(std::fabs(aveuu(i, j, k) - aveu(i, j, k) * aveu(i, j, k)));
                    avevv(i, j, k) = std::sqrt(std::fabs(avevv(i, j, k) - avev(i, j, k) * avev(i, j, k)));
                    aveww(i, j, k) = std::sqrt(std::fabs(aveww(i, j, k) - avew(i, j, k) * avew(i, j, k)));
                }
        for (int k = 1; k <= km; ++k)
            for (int i = 1; i <= im; ++i) {
                avesuu(i, k, 1) = std::sqrt(std::fabs(avesuu(i, k, 1) - avesu(i, k, 1) * avesu(i, k, 1)));
                avesvv(i, k, 1) = std::sqrt(std::fabs(avesvv(i, k, 1) - avesv(i, k, 1) * avesv(i, k, 1)));
                avesww(i, k, 1) = std::sqrt(std::fabs(avesww(i, k, 1) - avesw(i, k, 1) * avesw(i, k, 1)));
            }
    }
}

// bondFG.f95:15-31
void oracle_bondfg(int km, int jm, float *f_, int im, float *g_, float *h_) {
    const int ip = im, jp = jm, kp = km;
    A3 f = ARR_F(f_), g = ARR_F(g_), h = ARR_F(h_);
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) f(0, j, k) = f(1, j, k);
    for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) g(i, 0, k) = g(i, jm, k);
    for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
            h(i, j, 0) = 0.0f;
            h(i, j, km) = 0.0f;
        }
}

// boundp.f95:5-21
void oracle_boundp2(int jm, int im, float *p_, int km) {
    const int ip = im, jp = jm, kp = km;
    A3 p = ARR_P(p_);
    for (int j = 0; j <= jm + 1; ++j)
        for (int i = 0; i <= im + 1; ++i) {
            p(i, j, 0) = p(i, j, 1);
            p(i, j, km + 1) = p(i, j, km);
        }
}

// boundp.f95:23-44
void oracle_boundp1(int km, int jm, float *p_, int im) {
    const int ip = im, jp = jm, kp = km;
    A3 p = ARR_P(p_);
    for (int k = 0; k <= km + 1; ++k)
        for (int j = 0; j <= jm + 1; ++j) {
            p(0, j, k) = p(1, j, k);
            p(im + 1, j, k) = p(im, j, k);
        }
    for (int k = 0; k <= km + 1; ++k)
        for (int i = 0; i <= im + 1; ++i) {
            p(i, 0, k) = p(i, jm, k);
            p(i, jm + 1, k) = p(i, 1, k);
        }
}

// press.f95:49-146
// FP64-refined press after the FP32 SOR (the CUDA path's les_refine.cuh):
// p64 = p; for m = 0..M: r = b - A p64 in FP64, A the operator the sweeps
// relax (boundp1/boundp2 neighbours) with its diagonal the sum of the six
// coefficients, b = rhs_raw - mu with mu the mean of rhs weighted by A's
// left null vector w = wx wy wz (w(q+1) cs(q+1) = w(q) cl(q) per axis); the
// relative residual and the stop test; if m < M and not stopped: A e = r by
// `inner` FP32 SOR iterations from e = 0 (press.f95:87-115 with rhs = (float)
// r, no rhsav, no stop test), p64 += e.  Then pav in FP64 and
// p = (float)(p64 - pav) with boundp1/boundp2.  Returns (float) pav.
// The spectral inner solve (inner = 0) for uniform x and y spacing, by
// direct sums: DCT-II along i, real DFT along j, one tridiagonal solve in k
// per mode (the (0,0) mode drops its last equation, e(km) = 0), then the
// inverse sums.  r and e are (im, jm, km) arrays, i fastest.
static void oracle_spectral_solve(int im, int jm, int km, double c2, double c3, const std::vector<double> &zsub,
                                  const std::vector<double> &zdiag, const std::vector<double> &zsup,
                                  const std::vector<double> &r, std::vector<double> &e) {
    const double pi = 3.14159265358979323846;
    const int jh = jm / 2 + 1;
    // cos(pi m (2i+1) / 2im), cos and sin(2 pi n j / jm)
    std::vector<double> cx((size_t)im * im), cy((size_t)jh * jm), sy((size_t)jh * jm);
    for (int m = 0; m < im; ++m)
        for (int i = 0; i < im; ++i) cx[(size_t)m * im + i] = std::cos(pi * m * (2 * i + 1) / (2.0 * im));
    for (int n = 0; n < jh; ++n)
        for (int j = 0; j < jm; ++j) {
            cy[(size_t)n * jm + j] = std::cos(2.0 * pi * n * j / jm);
            sy[(size_t)n * jm + j] = std::sin(2.0 * pi * n * j / jm);
        }
    auto R = [&](int i, int j, int k) { return r[(size_t)i + (size_t)im * (j + (size_t)jm * k)]; };
    std::vector<double> X((size_t)im * jm * km);  // [k][j][m]
#pragma omp parallel for schedule(static)
    for (int k = 0; k < km; ++k)
        for (int j = 0; j < jm; ++j)
            for (int m = 0; m < im; ++m) {
                double s = 0.0;
                for (int i = 0; i < im; ++i) s += R(i, j, k) * cx[(size_t)m * im + i];
                X[(size_t)m + (size_t)im * (j + (size_t)jm * k)] = s;
            }
    std::vector<double> Yr((size_t)im * jh * km), Yi(Yr.size());  // [k][n][m]
#pragma omp parallel for schedule(static)
    for (int k = 0; k < km; ++k)
        for (int n = 0; n < jh; ++n)
            for (int m = 0; m < im; ++m) {
                double sr = 0.0, si = 0.0;
                for (int j = 0; j < jm; ++j) {
                    const double x = X[(size_t)m + (size_t)im * (j + (size_t)jm * k)];
                    sr += x * cy[(size_t)n * jm + j];
                    si -= x * sy[(size_t)n * jm + j];
                }
                Yr[(size_t)m + (size_t)im * (n + (size_t)jh * k)] = sr;
                Yi[(size_t)m + (size_t)im * (n + (size_t)jh * k)] = si;
            }
#pragma omp parallel for schedule(static)
    for (int n = 0; n < jh; ++n)
        for (int m = 0; m < im; ++m) {
            const double lam = 2.0 * c2 * (std::cos(pi * m / im) - 1.0) + 2.0 * c3 * (std::cos(2.0 * pi * n / jm) - 1.0);
            const int kn = (m == 0 && n == 0) ? km - 1 : km;
            std::vector<double> cp(km), dr(km), di(km);
            for (int k = 0; k < kn; ++k) {
                const double a = k > 0 ? zsub[k] : 0.0, b = zdiag[k] + lam, c = (k < kn - 1) ? zsup[k] : 0.0;
                const double den = b - a * (k > 0 ? cp[k - 1] : 0.0);
                const size_t q = (size_t)m + (size_t)im * (n + (size_t)jh * k);
                cp[k] = c / den;
                dr[k] = (Yr[q] - a * (k > 0 ? dr[k - 1] : 0.0)) / den;
                di[k] = (Yi[q] - a * (k > 0 ? di[k - 1] : 0.0)) / den;
            }
            double xr = 0.0, xi = 0.0;
            for (int k = kn - 1; k >= 0; --k) {
                if (k < kn - 1) {
                    xr = dr[k] - cp[k] * xr;
                    xi = di[k] - cp[k] * xi;
                } else {
                    xr = dr[k];
                    xi = di[k];
                }
                const size_t q = (size_t)m + (size_t)im * (n + (size_t)jh * k);
                Yr[q] = xr;
                Yi[q] = xi;
            }
            if (kn < km) {
                const size_t q = (size_t)m + (size_t)im * (n + (size_t)jh * (km - 1));
                Yr[q] = 0.0;
                Yi[q] = 0.0;
            }
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < km; ++k)  // inverse real DFT along j (Hermitian extension)
        for (int j = 0; j < jm; ++j)
            for (int m = 0; m < im; ++m) {
                double s = 0.0;
                for (int n = 0; n < jh; ++n) {
                    const size_t q = (size_t)m + (size_t)im * (n + (size_t)jh * k);
                    const bool edge = (n == 0 || 2 * n == jm);
                    const double re = edge ? Yr[q] * cy[(size_t)n * jm + j]
                                           : Yr[q] * cy[(size_t)n * jm + j] - Yi[q] * sy[(size_t)n * jm + j];
                    s += (edge ? 1.0 : 2.0) * re;
                }
                X[(size_t)m + (size_t)im * (j + (size_t)jm * k)] = s / jm;
            }
    e.assign((size_t)im * jm * km, 0.0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < km; ++k)  // inverse DCT-II along i
        for (int j = 0; j < jm; ++j)
            for (int i = 0; i < im; ++i) {
                double s = X[(size_t)im * (j + (size_t)jm * k)];
                for (int m = 1; m < im; ++m)
                    s += 2.0 * X[(size_t)m + (size_t)im * (j + (size_t)jm * k)] * cx[(size_t)m * im + i];
                e[(size_t)i + (size_t)im * (j + (size_t)jm * k)] = s / im;
            }
}

static float oracle_refine_tail(int km, int jm, int im, float *p_, const float *rraw, double rav,
                                const float *dx1_, const float *dy1_, const float *dzn_, const float *cn1_,
                                const float *cn2l_, const float *cn2s_, const float *cn3l_, const float *cn3s_,
                                const float *cn4l_, const float *cn4s_, float omega) {
    const int ip = im, jp = jm, kp = km;
    A3 p = ARR_P(p_), cn1 = ARR_I(cn1_);
    A1 dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1);
    A1 cn2l = mk1(cn2l_, 1), cn2s = mk1(cn2s_, 1), cn3l = mk1(cn3l_, 1), cn3s = mk1(cn3s_, 1),
       cn4l = mk1(cn4l_, 1), cn4s = mk1(cn4s_, 1);
    const size_t n = (size_t)im * jm * km;
    auto at = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)); };
    auto weights = [](const A1 &cl, const A1 &cs, int nq) {
        std::vector<double> w(nq, 1.0);
        for (int q = 1; q < nq; ++q) w[q] = w[q - 1] * (double)cl(q) / (double)cs(q + 1);
        return w;
    };
    const std::vector<double> wx = weights(cn2l, cn2s, im), wy = weights(cn3l, cn3s, jm), wz = weights(cn4l, cn4s, km);
    double sw = 0.0, swr = 0.0;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                const double w = wx[i - 1] * wy[j - 1] * wz[k - 1];
                swr += w * (double)rraw[at(i, j, k)];
                sw += w;
            }
    const double mu = swr / sw;
    std::vector<double> p64(n);
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) p64[at(i, j, k)] = (double)p(i, j, k);
    std::vector<float> er_((size_t)(ip + 2) * (jp + 2) * (kp + 2), 0.0f), e_((size_t)(ip + 3) * (jp + 3) * (kp + 2));
    A3 er = ARR_RHS(er_.data()), e = ARR_P(e_.data());
    double bnorm2 = 0.0, rel = 0.0;
    bool stop = false;
    g_ref_done = 0;
    for (int m = 0; m <= g_ref_outer; ++m) {
        double r2 = 0.0, b2 = 0.0;
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    const int jn = (j == jm) ? 1 : j + 1, js = (j == 1) ? jm : j - 1;
                    const double pc = p64[at(i, j, k)];
                    const double pe = (i == im) ? pc : p64[at(i + 1, j, k)];
                    const double pw = (i == 1) ? pc : p64[at(i - 1, j, k)];
                    const double pn = p64[at(i, jn, k)], ps = p64[at(i, js, k)];
                    const double pu = (k == km) ? pc : p64[at(i, j, k + 1)];
                    const double pd = (k == 1) ? pc : p64[at(i, j, k - 1)];
                    const double c2l = cn2l(i), c2s = cn2s(i), c3l = cn3l(j), c3s = cn3s(j), c4l = cn4l(k),
                                 c4s = cn4s(k);
                    const double diag = ((((c2l + c2s) + c3l) + c3s) + c4l) + c4s;
                    double s = c2l * pe;
                    s = s + c2s * pw;
                    s = s + c3l * pn;
                    s = s + c3s * ps;
                    s = s + c4l * pu;
                    s = s + c4s * pd;
                    const double ap = s - pc * diag;
                    const double b = (double)rraw[at(i, j, k)] - mu;
                    const double r = b - ap;
                    er(i, j, k) = (float)r;
                    r2 += r * r;
                    b2 += b * b;
                }
        if (m == 0) bnorm2 = b2;
        rel = bnorm2 > 0.0 ? std::sqrt(r2 / bnorm2) : 0.0;
        if (m == 0) g_ref_out[2] = rel;
        g_ref_out[3] = rel;
        if (rel <= g_ref_tol) stop = true;
        if (stop || m == g_ref_outer) break;
        if (g_ref_inner == 0) {  // spectral: r in FP64, then p64 += e
            std::vector<double> rr(n), ee;
            for (int k = 1; k <= km; ++k)
                for (int j = 1; j <= jm; ++j)
                    for (int i = 1; i <= im; ++i) {
                        const int jn = (j == jm) ? 1 : j + 1, js = (j == 1) ? jm : j - 1;
                        const double pc = p64[at(i, j, k)];
                        const double pe = (i == im) ? pc : p64[at(i + 1, j, k)];
                        const double pw = (i == 1) ? pc : p64[at(i - 1, j, k)];
                        const double pn = p64[at(i, jn, k)], ps = p64[at(i, js, k)];
                        const double pu = (k == km) ? pc : p64[at(i, j, k + 1)];
                        const double pd = (k == 1) ? pc : p64[at(i, j, k - 1)];
                        const double c2l = cn2l(i), c2s = cn2s(i), c3l = cn3l(j), c3s = cn3s(j), c4l = cn4l(k),
                                     c4s = cn4s(k);
                        const double diag = ((((c2l + c2s) + c3l) + c3s) + c4l) + c4s;
                        double s = c2l * pe;
                        s = s + c2s * pw;
                        s = s + c3l * pn;
                        s = s + c3s * ps;
                        s = s + c4l * pu;
                        s = s + c4s * pd;
                        rr[at(i, j, k)] = ((double)rraw[at(i, j, k)] - mu) - (s - pc * diag);
                    }
            std::vector<double> zsub(km), zdiag(km), zsup(km);
            for (int k = 1; k <= km; ++k) {
                zsub[k - 1] = cn4s(k);
                zsup[k - 1] = cn4l(k);
                double d = -((double)cn4l(k) + (double)cn4s(k));
                if (k == 1) d += cn4s(k);
                if (k == km) d += cn4l(k);
                zdiag[k - 1] = d;
            }
            oracle_spectral_solve(im, jm, km, cn2l(1), cn3l(1), zsub, zdiag, zsup, rr, ee);
            for (size_t q = 0; q < n; ++q) p64[q] = p64[q] + ee[q];
            ++g_ref_done;
            continue;
        }
        std::fill(e_.begin(), e_.end(), 0.0f);
        for (int l = 1; l <= g_ref_inner; ++l) {
            for (int nrd = 0; nrd <= 1; ++nrd) {
                for (int k = 1; k <= km; ++k)
                    for (int j = 1; j <= jm; ++j)
                        for (int i = 1 + (k + j + nrd) % 2; i <= im; i += 2) {
                            const float reltmp =
                                omega * (cn1(i, j, k) * (cn2l(i) * e(i + 1, j, k) + cn2s(i) * e(i - 1, j, k) +
                                                         cn3l(j) * e(i, j + 1, k) + cn3s(j) * e(i, j - 1, k) +
                                                         cn4l(k) * e(i, j, k + 1) + cn4s(k) * e(i, j, k - 1) -
                                                         er(i, j, k)) -
                                         e(i, j, k));
                            e(i, j, k) = e(i, j, k) + reltmp;
                        }
                oracle_boundp1(km, jm, e_.data(), im);
            }
            oracle_boundp2(jm, im, e_.data(), km);
        }
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) p64[at(i, j, k)] = p64[at(i, j, k)] + (double)e(i, j, k);
        ++g_ref_done;
    }
    double num = 0.0, den = 0.0;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                const double w = (double)dx1(i) * (double)dy1(j) * (double)dzn(k);
                num += p64[at(i, j, k)] * w;
                den += w;
            }
    const double pav = num / den;
    g_ref_out[0] = rav;
    g_ref_out[1] = pav;
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) p(i, j, k) = (float)(p64[at(i, j, k)] - pav);
    oracle_boundp1(km, jm, p_, im);
    oracle_boundp2(jm, im, p_, km);
    return (float)pav;
}

int oracle_press_ex(int km, int jm, int im, float *rhs_, const float *u_, const float *dx1_,
                    const float *v_, const float *dy1_, const float *w_, const float *dzn_,
                    float *f_, float *g_, float *h_, float dt, const float *cn1_,
                    const float *cn2l_, float *p_, const float *cn2s_, const float *cn3l_,
                    const float *cn3s_, const float *cn4l_, const float *cn4s_, int nmaxp,
                    float pjuge, float omega, float *sor_out, float *rhsav_out, float *pav_out) {
    const int ip = im, jp = jm, kp = km;
    A3 rhs = ARR_RHS(rhs_), u = ARR_U(u_), v = ARR_U(v_), w = ARR_W(w_), f = ARR_F(f_),
       g = ARR_F(g_), h = ARR_F(h_), cn1 = ARR_I(cn1_), p = ARR_P(p_);
    A1 dx1 = mk1(dx1_, -1), dy1 = mk1(dy1_, 0), dzn = mk1(dzn_, -1);
    A1 cn2l = mk1(cn2l_, 1), cn2s = mk1(cn2s_, 1), cn3l = mk1(cn3l_, 1), cn3s = mk1(cn3s_, 1),
       cn4l = mk1(cn4l_, 1), cn4s = mk1(cn4s_, 1);
    const bool canon = !(g_red_mode & ORACLE_RED_F_RHSAV);      // rhsav and area
    const bool canon_sor = !(g_red_mode & ORACLE_RED_F_SOR);    // SOR residual
    const bool canon_pav = !(g_red_mode & ORACLE_RED_F_PAV);    // pav and pco

    oracle_bondfg(km, jm, f_, im, g_, h_);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
                rhs(i, j, k) = (-u(i - 1, j, k) + u(i, j, k)) / dx1(i) +
                               (-v(i, j - 1, k) + v(i, j, k)) / dy1(j) +
                               (-w(i, j, k - 1) + w(i, j, k)) / dzn(k);
                rhs(i, j, k) = (f(i, j, k) - f(i - 1, j, k)) / dx1(i) +
                               (g(i, j, k) - g(i, j - 1, k)) / dy1(j) +
                               (h(i, j, k) - h(i, j, k - 1)) / dzn(k) + rhs(i, j, k) / dt;
            }
    float rhsav;
    double rhsav64 = 0.0;
    const bool refine = g_ref_outer > 0;
    std::vector<float> rraw;  // rhs before the rhsav subtraction (refined press)
    if (refine) {
        rraw.resize((size_t)im * jm * km);
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) rraw[(i - 1) + (size_t)im * ((j - 1) + (size_t)jm * (k - 1))] = rhs(i, j, k);
    }
    if (canon) {
        const double num = canonical_sum3(
            im, jm, km, [&](int i, int j, int k) { return dx1(i) * dy1(j) * dzn(k) * rhs(i, j, k); });
        const double den =
            canonical_sum3(im, jm, km, [&](int i, int j, int k) { return dx1(i) * dy1(j) * dzn(k); });
        rhsav64 = num / den;
        rhsav = (float)rhsav64;
    } else {
        float s = 0.0f, area = 0.0f;
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    s = s + dx1(i) * dy1(j) * dzn(k) * rhs(i, j, k);
                    area = area + dx1(i) * dy1(j) * dzn(k);
                }
        rhsav = s / area;
        rhsav64 = (double)rhsav;
    }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) rhs(i, j, k) = rhs(i, j, k) - rhsav;

    // SOR, press.f95:87-115.  Within one colour every update reads only cells
    // of the other colour and ghost cells, so the in-place sweep is order
    // independent; reltmp^2 of each cell is kept for the residual sum.
    std::vector<float> r2((size_t)im * jm * km);
    A3 rr = mk(r2.data(), 1, im, 1, jm, 1, km);
    int l_exec = 0;
    float sor = 0.0f;
    for (int l = 1; l <= nmaxp; ++l) {
        l_exec = l;
        float sor32 = 0.0f;
        FixSum sfix;
        for (int nrd = 0; nrd <= 1; ++nrd) {
#pragma omp parallel for schedule(static)
            for (int k = 1; k <= km; ++k)
                for (int j = 1; j <= jm; ++j)
                    for (int i = 1 + (k + j + nrd) % 2; i <= im; i += 2) {
                        float reltmp = omega * (cn1(i, j, k) * (cn2l(i) * p(i + 1, j, k) +
                                                                cn2s(i) * p(i - 1, j, k) +
                                                                cn3l(j) * p(i, j + 1, k) +
                                                                cn3s(j) * p(i, j - 1, k) +
                                                                cn4l(k) * p(i, j, k + 1) +
                                                                cn4s(k) * p(i, j, k - 1) - rhs(i, j, k)) -
                                                p(i, j, k));
                        p(i, j, k) = p(i, j, k) + reltmp;
                        rr(i, j, k) = reltmp * reltmp;
                    }
            for (int k = 1; k <= km; ++k)
                for (int j = 1; j <= jm; ++j)
                    for (int i = 1 + (k + j + nrd) % 2; i <= im; i += 2) {
                        if (canon_sor) sfix.add(rr(i, j, k));
                        else sor32 = sor32 + rr(i, j, k);
                    }
            oracle_boundp1(km, jm, p_, im);
        }
        oracle_boundp2(jm, im, p_, km);
        sor = canon_sor ? (float)sfix.value() : sor32;
        if (sor < pjuge) break;
    }

    if (refine) {
        const float pav = oracle_refine_tail(km, jm, im, p_, rraw.data(), rhsav64, dx1_, dy1_, dzn_, cn1_, cn2l_,
                                             cn2s_, cn3l_, cn3s_, cn4l_, cn4s_, omega);
        if (sor_out) *sor_out = sor;
        if (rhsav_out) *rhsav_out = rhsav;
        if (pav_out) *pav_out = pav;
        return l_exec;
    }
    float pav;
    if (canon_pav) {
        const double num = canonical_sum3(
            im, jm, km, [&](int i, int j, int k) { return p(i, j, k) * dx1(i) * dy1(j) * dzn(k); });
        const double den =
            canonical_sum3(im, jm, km, [&](int i, int j, int k) { return dx1(i) * dy1(j) * dzn(k); });
        pav = (float)(num / den);
    } else {
        float s = 0.0f, pco = 0.0f;
        for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
                for (int i = 1; i <= im; ++i) {
                    s = s + p(i, j, k) * dx1(i) * dy1(j) * dzn(k);
                    pco = pco + dx1(i) * dy1(j) * dzn(k);
                }
        pav = s / pco;
    }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) p(i, j, k) = p(i, j, k) - pav;
    oracle_boundp1(km, jm, p_, im);
    oracle_boundp2(jm, im, p_, km);
    if (sor_out) *sor_out = sor;
    if (rhsav_out) *rhsav_out = rhsav;
    if (pav_out) *pav_out = pav;
    return l_exec;
}

int oracle_press(int km, int jm, int im, float *rhs, const float *u, const float *dx1,
                 const float *v, const float *dy1, const float *w, const float *dzn, float *f,
                 float *g, float *h, float dt, const float *cn1, const float *cn2l, float *p,
                 const float *cn2s, const float *cn3l, const float *cn3s, const float *cn4l,
                 const float *cn4s, int n, int nmax, float *sor_out, float *rhsav_out,
                 float *pav_out) {
    (void)n;
    (void)nmax;
    // press.f95:44-46: pjuge = 0.0001, nmaxp = 50, omega = 1.
    return oracle_press_ex(km, jm, im, rhs, u, dx1, v, dy1, w, dzn, f, g, h, dt, cn1, cn2l, p, cn2s,
                           cn3l, cn3s, cn4l, cn4s, 50, 0.0001f, 1.0f, sor_out, rhsav_out, pav_out);
}

}  // extern "C"

namespace {

struct Scratch {
    std::vector<float> cov[9], nou[9], diu[9], dfu1, dfv1, dfw1, fx, fy, fz;
    Scratch(int ip, int jp, int kp) {
        const size_t n15 = (size_t)(ip + 4) * (jp + 3) * (kp + 3);
        const size_t nd = (size_t)(ip + 3) * (jp + 3) * (kp + 3);
        for (int a = 0; a < 9; ++a) {
            const size_t n = (a == 0 || a == 4) ? n15 : nd;
            cov[a].assign(n, 0.0f);
            nou[a].assign(n, 0.0f);
            diu[a].assign(n, 0.0f);
        }
        dfu1.assign((size_t)(ip + 1) * jp * kp, 0.0f);
        dfv1.assign((size_t)ip * (jp + 1) * kp, 0.0f);
        dfw1.assign((size_t)ip * jp * kp, 0.0f);
        const size_t nf = (size_t)(ip + 1) * (jp + 1) * (kp + 1);
        fx.assign(nf, 0.0f);
        fy.assign(nf, 0.0f);
        fz.assign(nf, 0.0f);
    }
};

void call_velfg(const oracle_params *P, oracle_fields *F, Scratch &S) {
    oracle_velfg(P->kp, P->jp, P->ip, F->dx1, S.cov[0].data(), S.cov[1].data(), S.cov[2].data(),
                 S.dfu1.data(), S.diu[0].data(), S.diu[1].data(), F->dy1, S.diu[2].data(), F->dzn,
                 P->vn, F->f, S.cov[3].data(), S.cov[4].data(), S.cov[5].data(), S.dfv1.data(),
                 S.diu[3].data(), S.diu[4].data(), S.diu[5].data(), F->g, S.cov[6].data(),
                 S.cov[7].data(), S.cov[8].data(), S.dfw1.data(), S.diu[6].data(), S.diu[7].data(),
                 S.diu[8].data(), F->dzs, F->h, S.nou[0].data(), F->u, S.nou[4].data(), F->v,
                 S.nou[8].data(), F->w, S.nou[1].data(), S.nou[2].data(), S.nou[3].data(),
                 S.nou[5].data(), S.nou[6].data(), S.nou[7].data());
}
void call_feedbf(const oracle_params *P, oracle_fields *F, Scratch &S) {
    oracle_feedbf(P->kp, P->jp, P->ip, F->usum, F->u, F->bmask1, F->vsum, F->v, F->cmask1, F->wsum,
                  F->w, F->dmask1, P->alpha, P->dt, P->beta, S.fx.data(), S.fy.data(), S.fz.data(),
                  F->f, F->g, F->h);
}
void call_les(const oracle_params *P, oracle_fields *F, Scratch &S) {
    oracle_les(P->kp, F->delx1, F->dx1, F->dy1, F->dzn, P->jp, P->ip, S.diu[0].data(),
               S.diu[1].data(), S.diu[2].data(), S.diu[3].data(), S.diu[4].data(), S.diu[5].data(),
               S.diu[6].data(), S.diu[7].data(), S.diu[8].data(), F->sm, F->f, F->g, F->h);
}
void call_bondv1(const oracle_params *P, oracle_fields *F, int n) {
    if (F->wind_profile)
        oracle_bondv1_ext_wind_profile(P->jp, F->u, F->z2, F->dzn, F->v, F->w, P->kp, n, P->ip,
                                       P->dt, F->dxs, F->wind_profile);
    else
        oracle_bondv1(P->jp, F->u, F->z2, F->dzn, F->v, F->w, P->kp, n, P->ip, P->dt, F->dxs);
}

}  // namespace

extern "C" {

// ifdata.f95:250-284 with ICAL=0, IFBF=1, IADAM=0
void oracle_ifdata(const oracle_params *P, oracle_fields *F, int n) {
    Scratch S(P->ip, P->jp, P->kp);  // zero_arrays (cov, diu, nou, dfu1..)
    const int ip = P->ip, jp = P->jp, kp = P->kp;
    A3 f = ARR_F(F->f), g = ARR_F(F->g), h = ARR_F(F->h);
    for (int k = 0; k <= kp; ++k)
        for (int j = 0; j <= jp; ++j)
            for (int i = 0; i <= ip; ++i) f(i, j, k) = g(i, j, k) = h(i, j, k) = 0.0f;
    call_bondv1(P, F, n);
    oracle_boundp1(kp, jp, F->p, ip);
    oracle_boundp2(jp, ip, F->p, kp);
    call_velfg(P, F, S);
    call_feedbf(P, F, S);
    call_les(P, F, S);
}

void oracle_run_steps(const oracle_params *P, oracle_fields *F, int n0, int nsteps, int nmax,
                      int *sor_iters) {
    Scratch S(P->ip, P->jp, P->kp);
    for (int s = 0; s < nsteps; ++s) {
        const int n = n0 + s;
        oracle_velnw(P->kp, P->jp, P->ip, F->p, P->ro, F->dxs, F->u, P->dt, F->f, F->dys, F->v, F->g,
                     F->dzs, F->w, F->h);
        call_bondv1(P, F, n);
        call_velfg(P, F, S);
        call_feedbf(P, F, S);
        call_les(P, F, S);
        oracle_adam(n, nmax, F->fold, P->ip, P->jp, P->kp, F->gold, F->hold, F->f, F->g, F->h);
        float sor, rhsav, pav;
        int it = oracle_press_ex(P->kp, P->jp, P->ip, F->rhs, F->u, F->dx1, F->v, F->dy1, F->w,
                                 F->dzn, F->f, F->g, F->h, P->dt, F->cn1, F->cn2l, F->p, F->cn2s,
                                 F->cn3l, F->cn3s, F->cn4l, F->cn4s, P->nmaxp, P->pjuge, P->omega,
                                 &sor, &rhsav, &pav);
        if (sor_iters) sor_iters[s] = it;
    }
}

}  // extern "C"
