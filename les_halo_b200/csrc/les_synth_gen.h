// les_synth_gen.h -- the seeded synthetic-input generators behind
// les_synth.h, as plain host C++ (no CUDA).  liblesb200.so exports them as
// les_synth_*; the CPU oracle library compiles the same source, so a CPU
// run builds bit-identical inputs without loading the library under test.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "les_synth.h"

namespace les_synth_gen {

// SplitMix64 (Steele, Lea, Flood 2014).
struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }  // (0,1)
    int irange(int lo, int hi) { return lo + (int)(next() % (uint64_t)(hi - lo + 1)); }
};

// The 150x150x90 benchmark case: dx=dy=4 m, dz 2 m x1.05, 30% plan area,
// 8-24 m footprints, lognormal heights mean 20 m sigma_ln 0.5 in 4-80 m,
// u*=0.3, z0=0.1, kappa=0.4, +-2% frozen noise.
inline void defaults(les_synth_cfg *c, int ip, int jp, int kp, uint64_t seed) {
    std::memset(c, 0, sizeof *c);
    c->ip = ip;
    c->jp = jp;
    c->kp = kp;
    c->dx = 4.0f;
    c->dy = 4.0f;
    c->dz0 = 2.0f;
    c->dz_growth = 1.05f;
    c->plan_area = 0.30f;
    c->foot_min = 2;
    c->foot_max = 6;
    c->h_mean = 20.0f;
    c->h_sigma_ln = 0.5f;
    c->h_min = 4.0f;
    c->h_max = 80.0f;
    c->ustar = 0.3f;
    c->z0 = 0.1f;
    c->kappa = 0.4f;
    c->noise = 0.02f;
    c->seed = seed;
}

// Uniform dx1(-1:ip+1), dy1(0:jp+1); dzn(1) = dz0 and dzn(k) = dzn(k-1) *
// growth for k = 2..kp+1 (dzn passed with its -1:kp+2 bounds).  The metric
// derivation of grid.f95:55-82 follows separately.
inline void base_grid(const les_synth_cfg *c, float *dx1, float *dy1, float *dzn) {
    for (int i = -1; i <= c->ip + 1; ++i) dx1[i + 1] = c->dx;
    for (int j = 0; j <= c->jp + 1; ++j) dy1[j] = c->dy;
    dzn[1 + 1] = c->dz0;
    for (int k = 2; k <= c->kp + 1; ++k) dzn[k + 1] = dzn[k] * c->dz_growth;
}

// Building heights zbm(-1:ip+1,-1:jp+1): rectangles placed until the plan
// area fraction is built (periodic in j, a margin in i); returns the built
// fraction.
inline float terrain(const les_synth_cfg *c, float *zbm) {
    const int ip = c->ip, jp = c->jp;
    const size_t ni = ip + 3;
    std::memset(zbm, 0, sizeof(float) * ni * (jp + 3));
    auto Z = [&](int i, int j) -> float & { return zbm[(size_t)(i + 1) + ni * (size_t)(j + 1)]; };
    SplitMix64 rng{c->seed ^ 0x5445525241494eull};
    const int margin = std::max(2, ip / 16);
    const long long target = (long long)std::ceil((double)c->plan_area * ip * jp);
    long long built = 0;
    const double sig = c->h_sigma_ln, mu = std::log((double)c->h_mean) - 0.5 * sig * sig;
    const int ilo = 1 + margin, ihi = ip - margin;
    for (int tries = 0; built < target && tries < 1000000; ++tries) {
        const int wx = rng.irange(c->foot_min, c->foot_max), wy = rng.irange(c->foot_min, c->foot_max);
        if (ihi - ilo + 1 < wx) break;
        const int i0 = rng.irange(ilo, ihi - wx + 1), j0 = rng.irange(1, jp);
        const double u1 = rng.uniform(), u2 = rng.uniform();
        const double nrm = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
        double hgt = std::exp(mu + sig * nrm);
        hgt = std::min<double>(std::max<double>(hgt, c->h_min), c->h_max);
        for (int j = j0; j < j0 + wy; ++j)
            for (int i = i0; i < i0 + wx; ++i) {
                const int jj = 1 + (j - 1) % jp;  // periodic in j
                float &z = Z(i, jj);
                if (z == 0.0f) ++built;
                z = std::max(z, (float)hgt);
            }
    }
    return (float)((double)built / ((double)ip * jp));
}

// wind_profile(1:jp,1:kp) = (u*/kappa) ln(zc/z0) (1 + xi), zc = z2(k) +
// dzn(k)/2 (z2 from 1, dzn with its -1:kp+2 bounds), xi ~ U(-noise, noise).
inline void inflow(const les_synth_cfg *c, const float *z2, const float *dzn, float *wp) {
    SplitMix64 rng{c->seed ^ 0x494e464c4f57ull};
    for (int k = 1; k <= c->kp; ++k) {
        const float zc = z2[k - 1] + 0.5f * dzn[k + 1];
        const double base = ((double)c->ustar / c->kappa) * std::log((double)zc / c->z0);
        for (int j = 1; j <= c->jp; ++j) {
            const double xi = (2.0 * rng.uniform() - 1.0) * c->noise;
            wp[(size_t)(j - 1) + (size_t)c->jp * (k - 1)] = (float)(base * (1.0 + xi));
        }
    }
}

}  // namespace les_synth_gen
