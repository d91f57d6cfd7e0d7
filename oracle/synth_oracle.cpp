// synth_oracle.cpp -- TEST INFRASTRUCTURE: the seeded synthetic inputs of
// les_synth.h (the same generator source, les_synth_gen.h) with the grid
// metrics of the oracle's own grid.f95 restatement, so that CPU runs (the
// reference arm and CPU baseline of bench.py, the tests) build their cases
// without loading liblesb200.so.
#include "les_oracle.h"
#include "les_synth_gen.h"

extern "C" {

void oracle_synth_default(les_synth_cfg *cfg, int ip, int jp, int kp, uint64_t seed) {
    les_synth_gen::defaults(cfg, ip, jp, kp, seed);
}

void oracle_synth_grid(const les_synth_cfg *c, float *dx1, float *dxl, float *dy1, float *dyl, float *z2,
                       float *dzn, float *dzs, float *dxs, float *dys) {
    les_synth_gen::base_grid(c, dx1, dy1, dzn);
    oracle_grid_metrics(c->ip, c->jp, c->kp, dx1, dxl, dy1, dyl, z2, dzn, dzs, dxs, dys);
}

float oracle_synth_terrain(const les_synth_cfg *c, float *zbm) { return les_synth_gen::terrain(c, zbm); }

void oracle_synth_inflow(const les_synth_cfg *c, const float *z2, const float *dzn, float *wp) {
    les_synth_gen::inflow(c, z2, dzn, wp);
}

}  // extern "C"
