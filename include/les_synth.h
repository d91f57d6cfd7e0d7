/*
 * les_synth.h -- seeded synthetic inputs for the LES step (part of
 * liblesb200.so; host-only, needs no GPU).
 *
 * The reference reads building heights from src/GIS/Tokyo_20mgrid.txt
 * (feedbfm.f95:33-39) and uses a fixed 20 m grid (grid.f95).  Benchmarks
 * and tests use these generators instead: rectangular blocks with lognormal
 * heights on a uniform horizontal grid with a geometric vertical stretch,
 * and a log-law inflow with frozen noise, all from SplitMix64 streams so
 * every run and every implementation sees bit-identical inputs.
 */
#ifndef LES_SYNTH_H
#define LES_SYNTH_H
#include "les_abi.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct les_synth_cfg {
    int ip, jp, kp;
    float dx, dy;          /* horizontal spacing (m)                        */
    float dz0, dz_growth;  /* dzn(1) and the geometric ratio for k=2..kp+1  */
    float plan_area;       /* target built fraction of columns (0..1)      */
    int foot_min, foot_max;/* building footprint edge, cells               */
    float h_mean, h_sigma_ln, h_min, h_max; /* lognormal heights (m)        */
    float ustar, z0, kappa, noise; /* log-law inflow and uniform noise     */
    uint64_t seed;
} les_synth_cfg;

/* Fill cfg with the 150x150x90 benchmark case (dx=dy=4 m, dz 2 m x1.05,
 * 30% plan area, 8-24 m footprints, lognormal heights mean 20 m sigma_ln
 * 0.5 clipped to 4-80 m, u*=0.3, z0=0.1, kappa=0.4, +-2% noise). */
void les_synth_default(les_synth_cfg *cfg, int ip, int jp, int kp, uint64_t seed);

/* dx1(-1:ip+1), dy1(0:jp+1), dzn(-1:kp+2) and the derived metrics
 * (les_grid_metrics). */
les_status les_synth_grid(const les_synth_cfg *cfg, float *dx1, float *dxl, float *dy1, float *dyl,
                          float *z2, float *dzn, float *dzs, float *dxs, float *dys);
/* Building heights zbm(-1:ip+1,-1:jp+1); returns the built fraction. */
float les_synth_terrain(const les_synth_cfg *cfg, float *zbm);
/* wind_profile(1:jp,1:kp) = (ustar/kappa) ln(zc/z0) (1+xi), zc = z2(k)+dzn(k)/2. */
les_status les_synth_inflow(const les_synth_cfg *cfg, const float *z2, const float *dzn,
                            float *wind_profile);

#ifdef __cplusplus
}
#endif
#endif
