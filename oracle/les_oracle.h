/*
 * les_oracle.h -- CPU restatement of the LES_Halo Fortran time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * les_halo_b200: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py load it.  The product never links or calls it.
 *
 * Every routine takes Fortran-layout (column-major) float arrays with exactly
 * the bounds the reference declares (src/Fortran/main_ocl.f95:41-167), passed
 * as the address of their first element, in the reference's argument order.
 * ip=im, jp=jm, kp=km (the reference aborts otherwise, ifdata.f95:216-219).
 *
 * Arithmetic is IEEE single precision, evaluated left to right in the order
 * the Fortran source writes it, compiled without FMA contraction.  Global sums
 * (rhsav, pav, the SOR residual) have two modes:
 *   ORACLE_RED_CANONICAL (default): each FP32 term is converted exactly to
 *       a Q63.64 fixed-point integer (truncated below 2^-64) and the terms
 *       are summed exactly in 128 bits, then finished in FP64.  The sum does
 *       not depend on order, and the CUDA path uses the same definition, so
 *       parity is bit-exact whatever reduction tree the kernels use.
 *   ORACLE_RED_FAITHFUL: the reference's sequential FP32 sums, in the
 *       Fortran loop order (press.f95:66-75 rhsav and area, 91-99 the SOR
 *       residual colour by colour, 127-133 pav and pco).
 * The mode is a bit mask: ORACLE_RED_F_RHSAV, ORACLE_RED_F_SOR and
 * ORACLE_RED_F_PAV make one sum faithful each (FAITHFUL = all three), so
 * the effect of each sum on the fields can be measured on its own.
 * Parity status: halo pack/unpack is pinned against the reference's own C
 * programs (src/OpenCL/test_halo_*.c); the physics fields are "parity
 * unpinned" because the reference ships no stored field values and no Fortran
 * compiler exists here to run it.
 */
#ifndef LES_ORACLE_H
#define LES_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORACLE_RED_CANONICAL = 0,
    ORACLE_RED_F_RHSAV = 1,
    ORACLE_RED_F_SOR = 2,
    ORACLE_RED_F_PAV = 4,
    ORACLE_RED_FAITHFUL = 7
};

void oracle_set_reduction_mode(int mode);
int oracle_get_reduction_mode(void);
/* FP64-refined press (the CUDA path's les_press_refine_fp64): outer = 0 is
 * the plain press.  oracle_last_refine fills rhsav, pav, rel_initial,
 * rel_final of the last press and returns the corrections applied. */
void oracle_set_press_refine(int outer, int inner, double tol);
int oracle_last_refine(double *out4);

/* set.f95:76-82 physical constants (vn computed as the Fortran does). */
void oracle_constants(float *ro, float *vn, float *alpha, float *beta);

/* grid.f95:22-82: the reference's 20 m grid (dx1=dy1=20, 3-segment dz). */
void oracle_grid_reference(int ip, int jp, int kp, float *dx1, float *dxl, float *dy1, float *dyl,
                           float *z2, float *dzn, float *dzs, float *dxs, float *dys);
/* grid.f95:55-82 metric derivation from given dx1(-1:ip+1), dy1(0:jp+1) and
 * dzn(1:kp+1) (dzn passed with its full -1:kp+2 bounds; entries 1..kp+1 are
 * read, the rest are written by the edge rules of grid.f95:60-65). */
void oracle_grid_metrics(int ip, int jp, int kp, float *dx1, float *dxl, float *dy1, float *dyl,
                         float *z2, float *dzn, float *dzs, float *dxs, float *dys);

/* init.f95:46-107 (zero u,v,w,p; masks via feedbfm; Poisson coefficients). */
void oracle_init(int km, int jm, int im, float *u, float *v, float *w, float *p, float *cn2s,
                 const float *dxs, float *cn2l, float *cn3s, const float *dys, float *cn3l,
                 const float *dzs, float *cn4s, float *cn4l, float *cn1, float *amask1,
                 float *bmask1, float *cmask1, float *dmask1, const float *zbm, const float *z2,
                 const float *dzn);
/* feedbfm.f95:21-63 with zbm(-1:ip+1,-1:jp+1) given (file read replaced). */
void oracle_feedbfm(int km, int jm, int im, float *amask1, float *bmask1, float *cmask1,
                    float *dmask1, const float *zbm, const float *z2, const float *dzn);

/* initial_wind_profile.f95 (power law, k<=78, k>=79 copies k=77). */
void oracle_initial_wind_profile(float *wind_profile, int jm, int km, const float *z2,
                                 const float *dzn);

void oracle_velnw(int km, int jm, int im, const float *p, float ro, const float *dxs, float *u,
                  float dt, const float *f, const float *dys, float *v, const float *g,
                  const float *dzs, float *w, const float *h);
void oracle_bondv1(int jm, float *u, const float *z2, const float *dzn, float *v, float *w, int km,
                   int n, int im, float dt, const float *dxs);
void oracle_bondv1_ext_wind_profile(int jm, float *u, const float *z2, const float *dzn, float *v,
                                    float *w, int km, int n, int im, float dt, const float *dxs,
                                    const float *wind_profile);
/* uout of the last bondv1 call (bondv1.f95:67-75), for inspection. */
float oracle_last_uout(void);

void oracle_vel2(int km, int jm, int im, float *nou1, const float *u, float *diu1, const float *dx1,
                 float *nou5, const float *v, float *diu5, const float *dy1, float *nou9,
                 const float *w, float *diu9, const float *dzn, float *cov1, float *cov5,
                 float *cov9, float *nou2, float *diu2, float *cov2, float *nou3, float *diu3,
                 const float *dzs, float *cov3, float *nou4, float *diu4, float *cov4, float *nou6,
                 float *diu6, float *cov6, float *nou7, float *diu7, float *cov7, float *nou8,
                 float *diu8, float *cov8);
void oracle_velfg(int km, int jm, int im, const float *dx1, float *cov1, float *cov2, float *cov3,
                  float *dfu1, float *diu1, float *diu2, const float *dy1, float *diu3,
                  const float *dzn, float vn, float *f, float *cov4, float *cov5, float *cov6,
                  float *dfv1, float *diu4, float *diu5, float *diu6, float *g, float *cov7,
                  float *cov8, float *cov9, float *dfw1, float *diu7, float *diu8, float *diu9,
                  const float *dzs, float *h, float *nou1, const float *u, float *nou5,
                  const float *v, float *nou9, const float *w, float *nou2, float *nou3,
                  float *nou4, float *nou6, float *nou7, float *nou8);
void oracle_feedbf(int km, int jm, int im, float *usum, const float *u, const float *bmask1,
                   float *vsum, const float *v, const float *cmask1, float *wsum, const float *w,
                   const float *dmask1, float alpha, float dt, float beta, float *fx, float *fy,
                   float *fz, float *f, float *g, float *h);
void oracle_les(int km, float *delx1, const float *dx1, const float *dy1, const float *dzn, int jm,
                int im, const float *diu1, const float *diu2, const float *diu3, const float *diu4,
                const float *diu5, const float *diu6, const float *diu7, const float *diu8,
                const float *diu9, float *sm, float *f, float *g, float *h);
void oracle_boundsm(int km, int jm, float *sm, int im);
void oracle_adam(int n, int nmax, float *fold, int im, int jm, int km, float *gold, float *hold,
                 float *f, float *g, float *h);
void oracle_bondfg(int km, int jm, float *f, int im, float *g, float *h);
/* aveflow.f95:42-157 (no file output).  aveu..uwfx (ip,jp,kp); avesu..avesww,
 * uwfxs (ip,kp); u, v, w, p, sm with the main_ocl.f95 bounds. */
void oracle_aveflow(int n, int n1, int km, int jm, int im, float *aveu, float *avev, float *avew,
                    float *avep, float *avel, float *aveuu, float *avevv, float *aveww, float *avesm,
                    float *avesmsm, float *uwfx, float *avesu, float *avesv, float *avesw,
                    float *avesuu, float *avesvv, float *avesww, const float *u, const float *v,
                    const float *w, const float *p, const float *sm, int nmax, float *uwfxs);
void oracle_boundp1(int km, int jm, float *p, int im);
void oracle_boundp2(int jm, int im, float *p, int km);
/* press.f95:49-146 (the I/O and print branches are omitted). Returns the
 * number of SOR iterations executed; *sor_out, *rhsav_out, *pav_out report
 * the final residual sum and the two means. */
int oracle_press(int km, int jm, int im, float *rhs, const float *u, const float *dx1,
                 const float *v, const float *dy1, const float *w, const float *dzn, float *f,
                 float *g, float *h, float dt, const float *cn1, const float *cn2l, float *p,
                 const float *cn2s, const float *cn3l, const float *cn3s, const float *cn4l,
                 const float *cn4s, int n, int nmax, float *sor_out, float *rhsav_out,
                 float *pav_out);
/* Same as oracle_press with the SOR sweep limit and tolerance given. */
int oracle_press_ex(int km, int jm, int im, float *rhs, const float *u, const float *dx1,
                    const float *v, const float *dy1, const float *w, const float *dzn, float *f,
                    float *g, float *h, float dt, const float *cn1, const float *cn2l, float *p,
                    const float *cn2s, const float *cn3l, const float *cn3s, const float *cn4l,
                    const float *cn4s, int nmaxp, float pjuge, float omega, float *sor_out,
                    float *rhsav_out, float *pav_out);

/* Whole-model state in Fortran layout, mirroring the arrays of main_ocl.f95. */
typedef struct oracle_fields {
    float *u, *v, *w, *p, *usum, *vsum, *wsum, *f, *g, *h, *fold, *gold, *hold, *rhs, *sm;
    float *amask1, *bmask1, *cmask1, *dmask1;
    float *cn1, *cn2l, *cn2s, *cn3l, *cn3s, *cn4l, *cn4s;
    float *dx1, *dy1, *dzn, *dzs, *dxs, *dys, *z2, *delx1;
    float *wind_profile; /* NULL: bondv1 power law; else bondv1_ext_wind_profile */
} oracle_fields;

typedef struct oracle_params {
    int ip, jp, kp;
    float dt, ro, vn, alpha, beta;
    int nmaxp;
    float pjuge, omega;
} oracle_params;

/* ifdata.f95:250-284 (ICAL=0, IFBF=1, IADAM=0): zero arrays, bondv1(n),
 * boundp1/2, velfg, feedbf, les.  zbm is not needed: the masks feedbfm
 * recomputes there are the ones already in fields. */
void oracle_ifdata(const oracle_params *prm, oracle_fields *fld, int n);
/* main_ocl.f95:233-299 for n = n0 .. n0+nsteps-1.  sor_iters (may be NULL)
 * receives the executed SOR iteration count of each step. */
void oracle_run_steps(const oracle_params *prm, oracle_fields *fld, int n0, int nsteps, int nmax,
                      int *sor_iters);

/* Canonical (exact fixed-point, FP64-finished) sum of one FP32 value per
 * interior cell (exposed for tests). */
double oracle_canonical_sum(int im, int jm, int km, const float *cell_values_ijk);

#ifdef __cplusplus
}
#endif
#endif
