/*
 * les_abi.h -- C ABI of liblesb200.so, the B200 (sm_100a) LES time step.
 *
 * Drop-in boundary for the LES_Halo reference (Hallot/LES_Halo):
 *   - a context API that replaces the accelerator driver pair
 *     initialise_LES_kernel / run_LES_kernel
 *     (src/OpenCL/module_LES_combined_ocl_TEMPL_V2.f95:18-30 and :219-231);
 *   - per-routine entry points with the Fortran argument order of the CPU
 *     routines called from src/Fortran/main_ocl.f95:264-299, so a Fortran
 *     host binds them with bind(C) interfaces (all scalars by reference);
 *   - halo pack/unpack entry points with the semantics of
 *     src/OpenCL/Kernels/halo_exchange.cl (and halo_exchange_correct.cl).
 *
 * Arrays crossing this boundary are host arrays in the reference's Fortran
 * layout (column-major, the bounds of main_ocl.f95:41-167 with ip=im, jp=jm,
 * kp=km), passed as the address of their first element, unless a function
 * says it takes device pointers.  The library owns all device memory; it
 * never keeps a caller's pointer beyond the call.  Every function returns a
 * les_status; none exits the process.  A context is not thread-safe; distinct
 * contexts are independent.  There is no CPU fallback: without a usable
 * B200 every compute call returns LES_ERR_CUDA.
 */
#ifndef LES_ABI_H
#define LES_ABI_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef enum les_status {
    LES_OK = 0,
    LES_ERR_BAD_ARG = 1, /* null pointer, bad size, bad mode            */
    LES_ERR_DIMS = 2,    /* grid extents unsupported (ifdata.f95:216)   */
    LES_ERR_CUDA = 3,    /* CUDA runtime error or no usable device      */
    LES_ERR_TIMEOUT = 4, /* a bounded device wait gave up               */
    LES_ERR_NAN = 5,     /* non-finite value found by a checking call   */
    LES_ERR_NOMEM = 6,   /* device allocation failed                    */
    LES_ERR_STATE = 7,   /* call out of order (e.g. step before upload) */
    LES_ERR_IO = 8       /* file missing, unreadable or of the wrong shape */
} les_status;

/* Last error message of the calling thread ("" after success). */
const char *les_last_error_string(void);
/* Library version string and the device the library runs on. */
const char *les_version(void);

/* Inflow modes of bondv1 (bondv1.f95:26-45 power law, or
 * bondv1_ext_wind_profile.f95:27-35 with an external wind_profile(jp,kp)). */
enum { LES_INFLOW_POWER_LAW = 0, LES_INFLOW_EXTERNAL = 1 };

typedef struct les_params {
    int ip, jp, kp;     /* interior extents (im, jm, km)                       */
    float dt;           /* set.f95:76                                          */
    float ro, vn;       /* set.f95:78-79                                       */
    float alpha, beta;  /* IBM feedback gains, set.f95:81-82                  */
    float cs0;          /* Smagorinsky constant, les.f95:123 (0.1)            */
    int nmaxp;          /* SOR iteration cap, press.f95:108 (50)               */
    float pjuge;        /* SOR stop threshold on sum(reltmp^2), press.f95:107  */
    float omega;        /* SOR relaxation, press.f95:109 (1.0)                 */
    int inflow_mode;    /* LES_INFLOW_*                                        */
    int ical;           /* 0: n==1 broadcast of the inflow plane (ICAL=0)      */
} les_params;

/* Fill p with the reference's constants for an ip x jp x kp grid
 * (set.f95:76-82, les.f95:123, press.f95:107-109; vn = 15.83*10.**(-6.)). */
les_status les_params_default(les_params *p, int ip, int jp, int kp);

/* Host arrays in Fortran layout (bounds as in main_ocl.f95). */
typedef struct les_host_fields {
    float *u, *v, *w;          /* (0:ip+1,-1:jp+1,0:kp+1), w (...,-1:kp+1) */
    float *p;                  /* (0:ip+2,0:jp+2,0:kp+1)                   */
    float *usum, *vsum, *wsum; /* (0:ip,0:jp,0:kp)                         */
    float *f, *g, *h;          /* (0:ip,0:jp,0:kp)                         */
    float *fold, *gold, *hold; /* (1:ip,1:jp,1:kp)                         */
    float *rhs;                /* (0:ip+1,0:jp+1,0:kp+1)                   */
    float *sm;                 /* (-1:ip+1,-1:jp+1,0:kp+1)                 */
    float *amask1, *dmask1;    /* (0:ip+1,0:jp+1,0:kp+1)                   */
    float *bmask1;             /* (-1:ip+1,0:jp+1,0:kp+1)                  */
    float *cmask1;             /* (0:ip+1,-1:jp+1,0:kp+1)                  */
    float *cn1;                /* (1:ip,1:jp,1:kp)                         */
    float *cn2l, *cn2s;        /* (ip)                                     */
    float *cn3l, *cn3s;        /* (jp)                                     */
    float *cn4l, *cn4s;        /* (kp)                                     */
    float *dx1;                /* (-1:ip+1)                                */
    float *dy1;                /* (0:jp+1)                                 */
    float *dzn, *dzs;          /* (-1:kp+2)                                */
    float *dxs;                /* (0:ip)                                   */
    float *dys;                /* (0:jp)                                   */
    float *z2;                 /* (1:kp+2)                                 */
    float *delx1;              /* (1:kp), output of les (may be NULL)       */
    float *wind_profile;       /* (1:jp,1:kp), LES_INFLOW_EXTERNAL only     */
} les_host_fields;

/* Per-step record (device-side values copied back by les_last_metrics). */
typedef struct les_metrics {
    int n;             /* time step index of the last step          */
    int sor_iters;     /* SOR iterations executed in that step       */
    float sor;         /* final sum(reltmp^2) (FP64 sum, rounded)   */
    float rhsav;       /* volume mean removed from rhs              */
    float pav;         /* volume mean removed from p                */
    float uout;        /* advective outflow speed (bondv1.f95:75)   */
    float p_centre, u_centre, v_centre, w_centre; /* press.f95:183-187 probe */
} les_metrics;

/* ---- context API: replaces initialise_LES_kernel / run_LES_kernel ---- */
typedef struct les_ctx les_ctx;

les_status les_ctx_create(const les_params *prm, les_ctx **out);
les_status les_ctx_destroy(les_ctx *ctx);
/* initialise_LES_kernel (TEMPL:18-215): copy the model state, metrics,
 * masks and Poisson coefficients to the device.  Fields the model does not
 * read (rhs, delx1) may be NULL.  Every array given is scanned first: a NaN
 * or Inf anywhere returns LES_ERR_NAN naming the array and its Fortran
 * index, before anything reaches the device. */
les_status les_ctx_upload(les_ctx *ctx, const les_host_fields *hf);
/* Copy the device state back; any NULL pointer is skipped.  rhs is returned
 * after the rhsav subtraction (press.f95:80-82), as the reference holds it. */
les_status les_ctx_download(les_ctx *ctx, les_host_fields *hf);
/* ifdata.f95:250-284 (ICAL=0, IFBF=1, IADAM=0) on the device: zero f,g,h,
 * bondv1(n), boundp1/2, velfg, feedbf, les.  Call after les_ctx_upload. */
les_status les_ctx_warmup(les_ctx *ctx, int n);
/* run_LES_kernel (TEMPL:219-1072): nsteps time steps n0..n0+nsteps-1 of
 * velnw, bondv1, velfg, feedbf, les, adam, press (main_ocl.f95:264-299).
 * Asynchronous on the context stream; les_ctx_sync waits. */
les_status les_step(les_ctx *ctx, int n0, int nsteps);
/* Replace the external inflow profile wind_profile(1:jp,1:kp) (host array)
 * before the next step (run_LES_kernel's per-step wind_profile argument). */
les_status les_set_wind_profile(les_ctx *ctx, const float *wind_profile);
les_status les_ctx_sync(les_ctx *ctx);
les_status les_last_metrics(les_ctx *ctx, les_metrics *m);
/* The WV_DEBUG sums (velnw.f95:61-68, feedbf.f95:30-36,68-83, the sum(x)
 * of every state array): sums[f] = the sum of field f (LES_F_*) over its
 * Fortran bounds, rhs as les_ctx_download returns it, each an exact Q63.64
 * sum of the FP32 values rounded to FP64 (independent of the order and of
 * the device).  LES_NFIELDS doubles; synchronous. */
les_status les_ctx_field_sums(les_ctx *ctx, double *sums);
/* CUDA stream (cudaStream_t) the context launches on. */
void *les_ctx_stream(les_ctx *ctx);
/* Number of kernels the library launched on this context so far. */
uint64_t les_ctx_launch_count(les_ctx *ctx);
/* Per-step phase timing with CUDA events recorded inside the step graph on
 * the context stream: the next nslots steps each get their own events
 * (nslots = 0 turns timing off).  les_ctx_phase_times returns, for one
 * slot, in milliseconds: [0] velnw+bondv1, [1] velfg+feedbf+sm, [2] boundsm
 * + visc + adam, [3] rhs + rhsav, [4] gap, [5] the first SOR colour sweep
 * (one launch), [6] the rest of the SOR loop, [7] pav, [8] the whole step. */
les_status les_ctx_set_timing(les_ctx *ctx, int nslots);
/* Diagnostic: exact != 0 makes every following step run the SOR one colour
 * sweep at a time with materialised ghosts (boundp1 per colour, boundp2 per
 * iteration, press.f95:87-115) instead of the multi-iteration passes.  Both
 * give identical results; odd jp and a just-uploaded p whose ghosts are not
 * boundary-consistent always use the per-colour sweeps. */
les_status les_ctx_set_sor_path(les_ctx *ctx, int exact);
/* Bounds-checked build (liblesb200_checked.so, compiled with LES_CHECKED):
 * every box index of the time step's kernels is checked against its
 * allocation; an index outside it is counted, the first one's (i, j, k)
 * kept, and the access redirected (no fault, no trap).  Returns the count
 * and that index after synchronising the device; in the regular build it
 * returns LES_ERR_STATE. */
les_status les_bounds_violations(unsigned long long *count, int *first_ijk);
/* Order of the step's global sums.  LES_RED_CANONICAL (default): rhsav, the
 * SOR residual and pav are exact sums (each FP32 term converted exactly to
 * fixed point, summed without rounding, finished in FP64), the same whatever
 * the reduction tree.  Each LES_RED_F_* bit instead takes one of them as the
 * reference's sequential FP32 loop, term for term in its Fortran order:
 * rhsav and the volume (press.f95:66-75), the residual sum(reltmp^2) over
 * colour 0 then colour 1 (press.f95:87-99), pav and pco (press.f95:123-133).
 * Those sums run on one thread block (milliseconds each): a parity mode,
 * not a fast path.  LES_RED_F_SOR runs the SOR one colour sweep at a time.
 * Excludes the FP64-refined press (LES_ERR_STATE). */
enum { LES_RED_CANONICAL = 0, LES_RED_F_RHSAV = 1, LES_RED_F_SOR = 2, LES_RED_F_PAV = 4,
       LES_RED_FAITHFUL = 7 };
les_status les_ctx_set_reduction_mode(les_ctx *ctx, int mode);
/* SOR iterations one SOR kernel launch of the next step carries: 0.5 for a
 * colour sweep, 2 for a multi-iteration pass. */
float les_ctx_sor_iters_per_launch(les_ctx *ctx);
/* Iterations per pass and tile rows the autotuner chose for the
 * multi-iteration SOR (0, 0 before the first step that uses it). */
les_status les_ctx_sor_tile(les_ctx *ctx, int *iters_per_pass, int *tile_rows);
/* The full pass shape: tile columns and k chunks too. */
les_status les_ctx_sor_shape(les_ctx *ctx, int *iters_per_pass, int *tile_rows, int *tile_cols,
                             int *k_chunks);
/* Region rows per warp of the chosen pass (1, or 2 for one-iteration passes
 * with two rows per warp; 0 before the first step that uses a pass).
 * LES_SOR_TILE=T,rows,chunks[,rows per warp] forces a shape. */
les_status les_ctx_sor_rows(les_ctx *ctx, int *rows_per_warp);
les_status les_ctx_phase_times(les_ctx *ctx, int slot, float *ms, int n);

/* Device state access for callers that keep fields on the GPU.  The field
 * is stored in a padded box: element (i,j,k) of the interior-indexed field
 * lives at ptr + (i + ox) + si*((j + 1) + sj*(k + 1)) (floats), for
 * -1 <= i <= ip+2, -1 <= j <= jp+2, -1 <= k <= kp+2. */
enum {
    LES_F_U = 0, LES_F_V, LES_F_W, LES_F_P, LES_F_USUM, LES_F_VSUM, LES_F_WSUM,
    LES_F_F, LES_F_G, LES_F_H, LES_F_FOLD, LES_F_GOLD, LES_F_HOLD, LES_F_RHS,
    LES_F_SM, LES_F_AMASK, LES_F_BMASK, LES_F_CMASK, LES_F_DMASK, LES_NFIELDS
};
les_status les_ctx_field(les_ctx *ctx, int field, float **dptr, int *ox, int *si, int *sj,
                         int *sk);

/* Halo ring of the context state, in the reference's buffer layout
 * (north|south|west|east, h_w = 1, TEMPL:111-127): the state arrays are
 * exchanged as the reference's combined arrays p2 (float2, extents
 * ip+3,jp+3,kp+2), uvw (float4, ip+2,jp+3,kp+3), uvwsum and fgh (float4,
 * ip+1,jp+1,kp+1), fgh_old (float4, ip,jp,kp), rhs (float, ip+2,jp+2,kp+2)
 * and sm (float, ip+3,jp+3,kp+2) (LES_combined_kernel.cl:345-364).  Host
 * buffers; sizes from les_ctx_halo_floats. */
enum { LES_H_P = 0, LES_H_UVW, LES_H_UVWSUM, LES_H_FGH, LES_H_FGH_OLD, LES_H_RHS, LES_H_SM,
       LES_NHALOS };
size_t les_ctx_halo_floats(les_ctx *ctx, int which);
/* ST_HALO_READ_*: pack the ring of the state array into buf (host). */
les_status les_ctx_halo_read(les_ctx *ctx, int which, float *buf);
/* ST_HALO_WRITE_*: unpack buf (host) into the ring of the state array.
 * Components with no state behind them are ignored: the second component
 * of p2 (p2 reads as (p, p)), the fourth of the float4 arrays, and u, v at
 * uvw's k = -1 layer (convert_to_uvw, module_LES_conversions.f95:18-21,
 * reads them as 0). */
les_status les_ctx_halo_write(les_ctx *ctx, int which, const float *buf);

/* ---- halo pack/unpack on caller arrays (halo_exchange.cl) -------------
 * array holds vdim floats per point (vdim = 1, 2, 4 or 16; the reference's
 * float, float2, float4, float16) with extents im (fastest), jm, km; h_w is
 * the ring width.  buffer size: les_halo_buffer_floats().  `device` != 0
 * means both pointers are device pointers (launched on `stream`, a
 * cudaStream_t or NULL); otherwise they are host pointers. */
size_t les_halo_buffer_floats(unsigned im, unsigned jm, unsigned km, unsigned h_w, unsigned vdim,
                              int inner);
/* exchange_{1,2,4,16}_halo_read, halo_exchange.cl:156-291 */
les_status les_halo_pack(const float *array, float *buffer, unsigned im, unsigned jm, unsigned km,
                         unsigned h_w, unsigned vdim, int device, void *stream);
/* exchange_{1,2,4,16}_halo_write, halo_exchange.cl:3-152 */
les_status les_halo_unpack(float *array, const float *buffer, unsigned im, unsigned jm,
                           unsigned km, unsigned h_w, unsigned vdim, int device, void *stream);
/* halo_exchange_correct.cl read: the owned inner ring, N|S without corners */
les_status les_halo_pack_inner(const float *array, float *buffer, unsigned im, unsigned jm,
                               unsigned km, unsigned h_w, unsigned vdim, int device, void *stream);
/* halo_exchange_correct.cl write (N|S buffer index without the im*w term) */
les_status les_halo_unpack_inner(float *array, const float *buffer, unsigned im, unsigned jm,
                                 unsigned km, unsigned h_w, unsigned vdim, int device,
                                 void *stream);

/* The same four operations for one component width each, named after the
 * reference's kernels exchange_{1,2,4,16}_halo_read (pack) and
 * exchange_{1,2,4,16}_halo_write (unpack), halo_exchange.cl:3-291 and
 * halo_exchange_correct.cl (the _inner forms). */
les_status les_halo_pack_1(const float *array, float *buffer, unsigned im, unsigned jm,
                           unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_1(float *array, const float *buffer, unsigned im, unsigned jm,
                             unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_inner_1(const float *array, float *buffer, unsigned im, unsigned jm,
                                 unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_inner_1(float *array, const float *buffer, unsigned im, unsigned jm,
                                   unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_2(const float *array, float *buffer, unsigned im, unsigned jm,
                           unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_2(float *array, const float *buffer, unsigned im, unsigned jm,
                             unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_inner_2(const float *array, float *buffer, unsigned im, unsigned jm,
                                 unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_inner_2(float *array, const float *buffer, unsigned im, unsigned jm,
                                   unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_4(const float *array, float *buffer, unsigned im, unsigned jm,
                           unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_4(float *array, const float *buffer, unsigned im, unsigned jm,
                             unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_inner_4(const float *array, float *buffer, unsigned im, unsigned jm,
                                 unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_inner_4(float *array, const float *buffer, unsigned im, unsigned jm,
                                   unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_16(const float *array, float *buffer, unsigned im, unsigned jm,
                           unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_16(float *array, const float *buffer, unsigned im, unsigned jm,
                             unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_pack_inner_16(const float *array, float *buffer, unsigned im, unsigned jm,
                                 unsigned km, unsigned h_w, int device, void *stream);
les_status les_halo_unpack_inner_16(float *array, const float *buffer, unsigned im, unsigned jm,
                                   unsigned km, unsigned h_w, int device, void *stream);

/* ---- setup feeding the step (a14) ------------------------------------ */
/* grid.f95:55-82 metric derivation: given dx1(-1:ip+1), dy1(0:jp+1) and
 * dzn(1:kp+1) (in an array with bounds -1:kp+2), fill dxl, dyl, z2, the
 * dzn edge rules, dzs, dxs, dys.  grid.f95:42-43 sets z2(1)=dzn(1). */
les_status les_grid_metrics(int ip, int jp, int kp, float *dx1, float *dxl, float *dy1,
                            float *dyl, float *z2, float *dzn, float *dzs, float *dxs, float *dys);
/* init.f95:82-107 Poisson coefficients cn1..cn4s, computed on the device. */
les_status les_poisson_coeffs(int ip, int jp, int kp, const float *dxs, const float *dys,
                              const float *dzs, float *cn1, float *cn2l, float *cn2s, float *cn3l,
                              float *cn3s, float *cn4l, float *cn4s);
/* feedbfm.f95:21-63 masks from building heights zbm(-1:ip+1,-1:jp+1),
 * computed on the device; mask entries outside 1..ip,1..jp,1..kp are left
 * as the caller initialised them. */
les_status les_building_masks(int ip, int jp, int kp, const float *zbm, const float *z2,
                              const float *dzn, float *amask1, float *bmask1, float *cmask1,
                              float *dmask1);

/* ---- per-routine drop-in entries (Fortran order, scalars by reference) --
 * Each copies its host arrays to the device, runs the routine's kernels and
 * copies the intent(out/inout) arrays back.  An output the caller does not
 * need may be NULL (e.g. cov/nou/dfu1 scratch of velfg). */
/* velnw.f95:5 */
les_status les_velnw_(const int *km, const int *jm, const int *im, const float *p, const float *ro,
                      const float *dxs, float *u, const float *dt, const float *f, const float *dys,
                      float *v, const float *g, const float *dzs, float *w, const float *h);
/* bondv1.f95:5 */
les_status les_bondv1_(const int *jm, float *u, const float *z2, const float *dzn, float *v,
                       float *w, const int *km, const int *n, const int *im, const float *dt,
                       const float *dxs);
/* bondv1_ext_wind_profile.f95:5 */
les_status les_bondv1_ext_wind_profile_(const int *jm, float *u, const float *z2, const float *dzn,
                                        float *v, float *w, const int *km, const int *n,
                                        const int *im, const float *dt, const float *dxs,
                                        const float *wind_profile);
/* velFG.f95:6 (diu1..9 are produced; cov*, nou*, dfu1/dfv1/dfw1 too when
 * non-NULL) */
les_status les_velfg_(const int *km, const int *jm, const int *im, const float *dx1, float *cov1,
                      float *cov2, float *cov3, float *dfu1, float *diu1, float *diu2,
                      const float *dy1, float *diu3, const float *dzn, const float *vn, float *f,
                      float *cov4, float *cov5, float *cov6, float *dfv1, float *diu4, float *diu5,
                      float *diu6, float *g, float *cov7, float *cov8, float *cov9, float *dfw1,
                      float *diu7, float *diu8, float *diu9, const float *dzs, float *h,
                      float *nou1, const float *u, float *nou5, const float *v, float *nou9,
                      const float *w, float *nou2, float *nou3, float *nou4, float *nou6,
                      float *nou7, float *nou8);
/* feedbf.f95:5 */
les_status les_feedbf_(const int *km, const int *jm, const int *im, float *usum, const float *u,
                       const float *bmask1, float *vsum, const float *v, const float *cmask1,
                       float *wsum, const float *w, const float *dmask1, const float *alpha,
                       const float *dt, const float *beta, float *fx, float *fy, float *fz,
                       float *f, float *g, float *h);
/* les.f95:98 (diu1..9 as produced by velfg) */
les_status les_les_(const int *km, float *delx1, const float *dx1, const float *dy1,
                    const float *dzn, const int *jm, const int *im, const float *diu1,
                    const float *diu2, const float *diu3, const float *diu4, const float *diu5,
                    const float *diu6, const float *diu7, const float *diu8, const float *diu9,
                    float *sm, float *f, float *g, float *h);
/* boundsm.f95:5 */
les_status les_boundsm_(const int *km, const int *jm, float *sm, const int *im);
/* adam.f95:5 (the data21 file write is the caller's) */
les_status les_adam_(const int *n, const int *nmax, float *fold, const int *im, const int *jm,
                     const int *km, float *gold, float *hold, float *f, float *g, float *h);
/* press.f95:72 (the data20 write and prints are the caller's); sor_iters
 * (may be NULL) receives the executed SOR iteration count. */
les_status les_press_(const int *km, const int *jm, const int *im, float *rhs, const float *u,
                      const float *dx1, const float *v, const float *dy1, const float *w,
                      const float *dzn, float *f, float *g, float *h, const float *dt,
                      const float *cn1, const float *cn2l, float *p, const float *cn2s,
                      const float *cn3l, const float *cn3s, const float *cn4l, const float *cn4s,
                      const int *n, const int *nmax, int *sor_iters);
/* press.f95 in sub-steps (each copies in, runs on the device, copies out):
 * les_press_rhsav_: press.f95:49-82, bondfg, rhs, rhsav and rhs -= rhsav;
 *   rhsav (may be NULL) receives the average.
 * les_press_sor_sweep_: press.f95:89-98 for colour *nrd (0 or 1), the sweep
 *   then boundp1; rhs is the one press holds after the rhsav subtraction;
 *   sor (may be NULL) receives this colour's sum of reltmp^2 (exact sum,
 *   rounded once).
 * les_press_residual_: one SOR iteration, press.f95:87-103 (both colours,
 *   boundp1 after each, boundp2); sor receives the iteration's residual.
 * les_press_pav_adj_: press.f95:123-146, pav, p -= pav, boundp1, boundp2;
 *   pav (may be NULL) receives the average. */
les_status les_press_rhsav_(const int *km, const int *jm, const int *im, float *rhs, const float *u,
                            const float *dx1, const float *v, const float *dy1, const float *w,
                            const float *dzn, float *f, float *g, float *h, const float *dt,
                            float *rhsav);
les_status les_press_sor_sweep_(const int *km, const int *jm, const int *im, const float *rhs,
                                const float *cn1, const float *cn2l, float *p, const float *cn2s,
                                const float *cn3l, const float *cn3s, const float *cn4l,
                                const float *cn4s, const int *nrd, float *sor);
les_status les_press_residual_(const int *km, const int *jm, const int *im, const float *rhs,
                               const float *cn1, const float *cn2l, float *p, const float *cn2s,
                               const float *cn3l, const float *cn3s, const float *cn4l,
                               const float *cn4s, float *sor);
les_status les_press_pav_adj_(const int *km, const int *jm, const int *im, float *p, const float *dx1,
                              const float *dy1, const float *dzn, float *pav);
/* Adjoint (reverse mode) of press.f95:49-146 run with *niter SOR iterations
 * and relaxation factor *omega (the count les_press_ reported; with it fixed
 * press is linear in u, v, w, f, g, h and the initial p).  No counterpart in
 * the reference.  On entry rhsb, pb, fb, gb, hb hold the adjoints of press's
 * outputs rhs, p, f, g, h (same Fortran bounds as those arrays); on return
 * pb, fb, gb, hb hold the adjoints of its inputs p, f, g, h, rhsb that of its
 * input rhs (0 on the interior press overwrites), and the adjoints of u, v, w
 * are ADDED to ub, vb, wb.  dx1, dy1, dzn, dt, cn1..cn4s as given to press. */
les_status les_press_b_(const int *km, const int *jm, const int *im, float *rhsb, const float *dx1,
                        const float *dy1, const float *dzn, float *fb, float *gb, float *hb,
                        const float *dt, const float *cn1, const float *cn2l, float *pb,
                        const float *cn2s, const float *cn3l, const float *cn3s, const float *cn4l,
                        const float *cn4s, const int *niter, const float *omega, float *ub,
                        float *vb, float *wb);
/* Adjoints of velnw.f95:5, feedbf.f95:5 and adam.f95:5, same argument order
 * as the forward entries with each state array replaced by its adjoint (no
 * counterpart in the reference).  On entry an array holds the adjoint of the
 * routine's output of that name; on return the adjoint of its input.
 * Arrays that are inputs only (velnw: p, f, g, h; feedbf: u, v, w) have the
 * adjoint ADDED.  fxb..fzb may be NULL (no seed). */
les_status les_velnw_b_(const int *km, const int *jm, const int *im, float *pb, const float *ro,
                        const float *dxs, float *ub, const float *dt, float *fb, const float *dys,
                        float *vb, float *gb, const float *dzs, float *wb, float *hb);
les_status les_feedbf_b_(const int *km, const int *jm, const int *im, float *usumb, float *ub,
                         const float *bmask1, float *vsumb, float *vb, const float *cmask1,
                         float *wsumb, float *wb, const float *dmask1, const float *alpha,
                         const float *dt, const float *beta, float *fxb, float *fyb, float *fzb,
                         float *fb, float *gb, float *hb);
les_status les_adam_b_(const int *n, const int *nmax, float *foldb, const int *im, const int *jm,
                       const int *km, float *goldb, float *holdb, float *fb, float *gb, float *hb);
/* Adjoint of les.f95:98 at the forward state given by diu1..9 (no counterpart
 * in the reference): smb, fb, gb, hb hold the adjoints of les's outputs sm,
 * f, g, h; on return smb holds that of its input sm (0 where les overwrites
 * it), the adjoints of diu1..9 are ADDED to diu1b..diu9b, and those of f, g, h
 * equal fb, gb, hb (unchanged).  Where a cell's strain invariant is 0 no
 * derivative passes through its sqrt. */
les_status les_les_b_(const int *km, const float *dx1, const float *dy1, const float *dzn,
                      const int *jm, const int *im, const float *diu1, const float *diu2,
                      const float *diu3, const float *diu4, const float *diu5, const float *diu6,
                      const float *diu7, const float *diu8, const float *diu9, float *diu1b,
                      float *diu2b, float *diu3b, float *diu4b, float *diu5b, float *diu6b,
                      float *diu7b, float *diu8b, float *diu9b, float *smb, const float *fb,
                      const float *gb, const float *hb);
/* bondFG.f95:5 */
les_status les_bondfg_(const int *km, const int *jm, float *f, const int *im, float *g, float *h);
/* boundp.f95:36 */
les_status les_boundp1_(const int *km, const int *jm, float *p, const int *im);
/* boundp.f95:18 */
les_status les_boundp2_(const int *jm, const int *im, float *p, const int *km);

/* ---- press.f95:49-81 without allocating (no counterpart in the reference) --
 * bondfg, rhs, rhsav and rhs -= rhsav, as les_press_ computes them, on
 * arrays the caller already holds on the device (same Fortran layouts and
 * argument order as les_press_; scalars by value), enqueued on `stream`
 * (a cudaStream_t or NULL); rhsav (a device float, may be NULL) receives
 * the average.  For hosts that cannot allocate device memory in their time
 * loop: one whose memory pool already holds the free device memory (a
 * cudaMalloc would fail), or one that keeps other streams busy (cudaFree
 * synchronises the whole device).  Allocates no device memory: the
 * per-block partial sums sit in a 256 KiB static __device__ array that every
 * GPU loading the library holds until exit, so ceil(im/32) * ceil(jm/8) must be
 * at most 5456 (e.g. im = jm = 1024 needs 4096); larger grids are rejected
 * with LES_ERR_DIMS before any device work.  The first call on each device
 * looks up the scratch address; make it outside any stream capture.  The
 * address is kept for the life of the process, which assumes each device
 * keeps one primary context: after cudaDeviceReset (which unloads the
 * module holding the scratch) the kept address is stale, so do not call
 * this entry again in that process.  Calls that overlap in time on one
 * device share the scratch and race. */
les_status les_press_rhs_noalloc(int km, int jm, int im, float *rhs, const float *u,
                                 const float *dx1, const float *v, const float *dy1,
                                 const float *w, const float *dzn, float *f, float *g, float *h,
                                 float dt, float *rhsav, void *stream);

/* ---- Time statistics: aveflow.f95:5-179 ------------------------------------
 * The eleven (ip,jp,kp) arrays and seven (ip,kp) arrays of aveflow, Fortran
 * order, interior only.  A NULL member is skipped by upload/download. */
typedef struct les_aveflow_fields {
    float *aveu, *avev, *avew, *avep, *avel, *aveuu, *avevv, *aveww, *avesm, *avesmsm,
        *uwfx;                                                    /* (ip,jp,kp) */
    float *avesu, *avesv, *avesw, *avesuu, *avesvv, *avesww, *uwfxs; /* (ip,kp)    */
} les_aveflow_fields;

/* aveflow.f95:42-175 on the context's state after step n (call it after
 * les_step for n, as main_ocl.f95:313 calls aveflow after the step): at
 * n == n1 the sums restart, for n >= n1 u, v, w, p, sm, their squares and
 * the uw flux are added, and at n == nmax the means, rms values and j means
 * are formed and, for each non-NULL, non-blank file name, the data10 file
 * (n,time; aveu, avew, avev) and the data11 file (n,time; aveuu, aveww,
 * avevv, uwfx) are written as the reference writes them (gfortran
 * unformatted sequential records, big-endian).  The statistics stay on the
 * device (allocated and zeroed on the first call); uwfxs is accumulated
 * from its current value, as in the reference, which never zeroes it.
 * Bit-identical to the reference's loops except at k = 1 of the uwfx
 * finish (aveflow.f95:112), where the reference reads aveu and avew before
 * the start of the arrays; those values are taken as 0 here. */
les_status les_aveflow(les_ctx *ctx, int n, int n1, int nmax, float time, const char *data10,
                       const char *data11);
les_status les_aveflow_upload(les_ctx *ctx, const les_aveflow_fields *stats);
les_status les_aveflow_download(les_ctx *ctx, les_aveflow_fields *stats);
/* aveflow.f95:5 with its Fortran argument order (host arrays by reference;
 * data10/data11 are file names, NULL or blank for no file).  u, v, w use the
 * bounds of main_ocl.f95, p (0:ip+2,0:jp+2,0:kp+1), sm (-1:ip+1,-1:jp+1,0:kp+1). */
les_status les_aveflow_(const int *n, const int *n1, const int *km, const int *jm, const int *im,
                        float *aveu, float *avev, float *avew, float *avep, float *avel,
                        float *aveuu, float *avevv, float *aveww, float *avesm, float *avesmsm,
                        float *uwfx, float *avesu, float *avesv, float *avesw, float *avesuu,
                        float *avesvv, float *avesww, const float *u, const float *v,
                        const float *w, const float *p, const float *sm, const int *nmax,
                        float *uwfxs, const char *data10, const float *time, const char *data11);

/* ---- Restart files ----------------------------------------------------------
 * les_write_restart writes the reference's restart records from the
 * context's state: data20 = u, v, w, p, usum, vsum, wsum (press.f95:191-201,
 * write_uvw_p_uvwsum_to_file at module_LES_combined_ocl_TEMPL_V2.f95:1194)
 * and data21 = fold, gold, hold (write_fgh_old_to_file,
 * module_LES_combined_ocl_TEMPL_V2.f95:1217) plus fghold as a fourth record
 * when fghold is not NULL (adam.f95:22-31 writes four).  Interior
 * (1:ip,1:jp,1:kp) of each array, one record each, big-endian gfortran
 * unformatted.  The reference writes them when mod(n,1000) == 0 or n == nmax;
 * the caller decides.  A NULL or blank name skips that file.
 * les_read_restart is the ICAL=1 reader of ifdata.f95:227-247: data30 holds
 * (n,time) and then the seven data20 records, data31 the data21 records
 * (fghold, if requested, must be the fourth).  Both files are read and
 * checked before the device state changes; the interiors of u, v, w, p,
 * usum, vsum, wsum, fold, gold, hold are replaced and their ghosts kept.
 * Follow with les_ctx_warmup, as ifdata continues after reading. */
les_status les_write_restart(les_ctx *ctx, const char *data20, const char *data21,
                             const float *fghold);
les_status les_read_restart(les_ctx *ctx, const char *data30, const char *data31, int *n,
                            float *time, float *fghold);

/* ---- FP64-refined pressure solve (no counterpart in the reference) -------
 * outer > 0 turns it on for the following steps: after the plain FP32 SOR
 * of press.f95:87-115, up to `outer` FP64 defect corrections follow, each
 * r = b - A p64 in FP64 and A e = r, p64 += e, until ||r||2/||b||2 <= rel_tol.
 * A is the operator the sweeps relax with its diagonal the sum of its six
 * coefficients (exactly singular, like the Neumann/periodic problem), and
 * b = rhs minus the mean of rhs weighted by A's left null vector (so A e = b
 * is solvable; on a stretched grid the reference's rhsav weights are not that
 * vector).  inner > 0: A e = r by `inner` FP32 SOR iterations from e = 0
 * (needs even jp); inner = 0: an FP64 spectral solve (DCT-II in i, DFT in j,
 * tridiagonal in k; needs even ip and jp and uniform x and y spacing), which
 * solves A e = r to FP64 rounding, issued after the captured step graph with
 * one host synchronisation per correction (such contexts cannot join an
 * ensemble).  pav (press.f95:123-133) is then formed in FP64 and
 * p = (float)(p64 - pav) with its boundp1/boundp2 copies.  outer = 0
 * restores the plain press.
 * les_last_refine_metrics reports the last step's FP64 rhsav and pav, the
 * relative residual before the first and after the last correction, and
 * the corrections applied. */
typedef struct les_refine_metrics {
    double rhsav, pav, rel_initial, rel_final;
    int outer;
} les_refine_metrics;
les_status les_press_refine_fp64(les_ctx *ctx, int outer, int inner, double rel_tol);
les_status les_last_refine_metrics(les_ctx *ctx, les_refine_metrics *m);

/* ---- NetCDF output: src/OpenCL/module_LES_write_netcdf.f95 ------------------
 * les_netcdf_open is init_netcdf_file (:105-322): it creates
 * <prefix>LES_output.nc and LES_output_p.nc (pressure, hPa), LES_output_u/_v/_w.nc
 * (velocity_x/_y/_z, m/s) and LES_output_uvwsum.nc (velocity_sum_x/_y/_z),
 * each with dimensions level, latitude, longitude (the full Fortran extents of
 * its arrays, ghosts included: p (ip+3,jp+3,kp+2), u and v (ip+2,jp+3,kp+2),
 * w (ip+2,jp+3,kp+3), usum.. (ip+1,jp+1,kp+1)) and a time dimension of
 * `ntimes` slots (NTIMESTEPS = 20 in the reference), the coordinate variables
 * latitude, longitude (1..n) and time (1..ntimes) and their units.  prefix is
 * prepended to the file names (NULL: "./").  les_netcdf_write puts time slot t
 * (1-based; the reference passes n/1000) of the context's p, u, v, w, usum,
 * vsum, wsum (write_to_netcdf_file, :324-357); les_netcdf_write_host does the
 * same from host arrays with those Fortran bounds.  les_netcdf_close
 * (close_netcdf_file, :359-386) fills the slots never written with the
 * default float fill value and closes.  Classic format, 64-bit offsets when a
 * file reaches 2 GiB. */
typedef struct les_netcdf les_netcdf;
les_status les_netcdf_open(const char *prefix, int ip, int jp, int kp, int ntimes, les_netcdf **nc);
les_status les_netcdf_write(les_netcdf *nc, les_ctx *ctx, int t);
les_status les_netcdf_write_host(les_netcdf *nc, int t, const float *p, const float *u, const float *v,
                                 const float *w, const float *usum, const float *vsum,
                                 const float *wsum);
les_status les_netcdf_close(les_netcdf *nc);

/* ---- Batched ensemble: many domains, one graph launch per step -------------
 * The reference advances one domain per run (main_ocl.f95:232-317); an
 * ensemble of uneven domains is this library's addition.  Members are
 * ordinary contexts, created, uploaded and (optionally) warmed up by the
 * caller, each with its own grid, terrain, inflow and autotuned SOR pass
 * shape; the ensemble borrows them (destroy it before them).
 * les_ensemble_step advances every member from step n0 to n0+nsteps-1 with
 * one cudaGraphLaunch per step: each member's step is a branch of one
 * captured graph, so the members' kernels run concurrently.  Results equal
 * les_step on each member, bit for bit.  Work queued earlier on a member's
 * stream runs first, and work queued on it afterwards (downloads,
 * les_last_metrics, les_step) waits for the ensemble's steps. */
typedef struct les_ensemble les_ensemble;
les_status les_ensemble_create(int nmembers, les_ctx *const *members, les_ensemble **ens);
les_status les_ensemble_step(les_ensemble *ens, int n0, int nsteps);
les_status les_ensemble_sync(les_ensemble *ens);
void *les_ensemble_stream(les_ensemble *ens);
/* The ensemble autotuner's record (after the first les_ensemble_step): the
 * candidates' times in ms per four tuning passes of every member (cap
 * entries at most; -1 where not run), their count and the index chosen.
 * Candidate 0: each member's own shape; 1..9: one-iteration passes of
 * (tile rows, k chunks, region rows per warp) (28, 1, 1), (28, 2, 1),
 * (24, 1, 1), (20, 1, 1), (12, 1, 1), (28, 1, 2), (28, 2, 2), (20, 1, 2),
 * (12, 1, 2) where a member can run them.  LES_ENSEMBLE_TUNE=own skips the
 * tuner. */
les_status les_ensemble_tune_info(les_ensemble *ens, float *ms, int cap, int *ncand, int *chosen);
/* kernels launched by the ensemble so far (all members) */
uint64_t les_ensemble_launch_count(les_ensemble *ens);
les_status les_ensemble_destroy(les_ensemble *ens);

/* ---- Adjoint of whole time steps (no counterpart in the reference) --------
 * The discrete adjoint of the step run by les_step (velnw, bondv1 with the
 * external inflow profile, velfg, feedbf, les, adam, press with a fixed SOR
 * iteration count), in FP32 with FP64 parameter gradients, on the device
 * state of a context created with LES_INFLOW_EXTERNAL.  The caller drives
 * checkpointing and recomputation: state slots hold copies of the
 * context's state (u v w p usum vsum wsum f g h fold gold hold rhs sm), and
 * les_adj_step_b applies the adjoint of step n whose input state is in a
 * slot to the adjoint state the handle holds, recomputing the forward
 * values it needs (the velocities after velnw and after bondv1, vel2's diu,
 * les's sm, feedbf's force) from that slot.  Parameter gradients
 * accumulate: the inflow profile wind_profile(1:jp,1:kp) (held fixed over
 * the steps) and, with les_ctx_set_drag, the per-column force scale.
 *
 * les_ctx_set_drag: f += s(i,j) * fx in feedbf (and g, h alike) for the
 *   following steps (drag(1:ip,1:jp), host; NULL: s = 1, the reference).
 * les_adj_create: nslots state slots; niter is the SOR iteration count
 *   every differentiated step executes (run the forward with nmaxp = niter
 *   and a pjuge it never reaches, e.g. -1).  Call after les_ctx_upload;
 *   the grid tables must not change afterwards.
 * les_adj_save / les_adj_load: context state to / from a slot.
 * les_adj_zero: adjoint state and parameter gradients to zero.
 * les_adj_tke: J = mean over the cells of box {i0,i1,j0,j1,k0,k1}
 *   (inclusive, interior indices) of 0.5 (uc^2 + vc^2 + wc^2) with the
 *   cell-centred velocities of anime.f95:45-47, of a slot (-1: the
 *   context's state), in FP64.
 * les_adj_seed_tke: adjoint of u, v, w += scale * dJ/d(u, v, w) at a slot
 *   (-1: the context's state).
 * les_adj_step_b: the adjoint of step n (input state in slot); afterwards
 *   the adjoint state is that of the step's input.
 * les_adj_read: parameter gradients (FP64: wind_profile jp*kp, drag ip*jp)
 *   and the adjoint state (Fortran layouts); NULL pointers are skipped.
 * les_adj_write: set the adjoint state from host arrays (Fortran layouts;
 *   NULL: that array's adjoint is zero). */
typedef struct les_adj les_adj;
les_status les_ctx_set_drag(les_ctx *ctx, const float *drag);
les_status les_adj_create(les_ctx *ctx, int nslots, int niter, les_adj **out);
les_status les_adj_destroy(les_adj *adj);
les_status les_adj_save(les_adj *adj, int slot);
les_status les_adj_load(les_adj *adj, int slot);
les_status les_adj_zero(les_adj *adj);
les_status les_adj_tke(les_adj *adj, int slot, const int *box, double *J);
les_status les_adj_seed_tke(les_adj *adj, int slot, const int *box, double scale);
les_status les_adj_step_b(les_adj *adj, int n, int slot);
les_status les_adj_read(les_adj *adj, double *wind_profile_b, double *drag_b, les_host_fields *state_b);
les_status les_adj_write(les_adj *adj, const les_host_fields *state_b);

/* ---- x-decomposed domain (no reference counterpart: the reference
 * round-trips its halos through ST_HALO_READ_* / ST_HALO_WRITE_* states,
 * module_LES_combined_ocl_TEMPL_V2.f95:438-491, on one device).  One context
 * per rank holds a slab of columns, created and uploaded like any context
 * from the slab's arrays: columns olo..ohi are its own, the others (at most
 * H on each side) a copy of its neighbours' own columns.  The host drives
 * the step as phases and, between them, exchanges the halo columns
 * (les_dd_pack on the owner, les_dd_unpack on the neighbour) and sums the
 * limbs of les_dd_sums over the ranks (64-bit integer sums; NCCL all-reduce
 * or device copies).  Step n, with K = 1 when n == 1 and ical == 0, else 2:
 *   BEGIN(n); halo(u v w p f g h usum vsum wsum fold gold hold);
 *   MOMENTUM(K); sum; RHSAV; halo(rhs);
 *   nmaxp times: [every m-th iteration but the first: halo(p)]
 *                SOR_ITER; sum; SOR_TEST;
 *   PAV_SUM; sum; PAV_END.
 * With halo width H >= 12 and m <= H/2 every own cell equals the single
 * domain's bit for bit (canonical FP32 sums; the SOR on the one-iteration
 * pass kernels, or per colour with LES_DD_SOR=colour).
 * les_dd_area_part: this rank's share (own columns) of the rhsav / pav
 *   denominator as an exact Q63.64 sum (lo, hi, bad); the ranks add the
 *   128-bit values and pass the total to les_dd_set_owned.
 * les_dd_set_owned: make the context a rank: own columns olo..ohi (the
 *   global sums count only these) and the whole domain's denominator.
 *   les_step then refuses the context.
 * les_dd_block_floats: floats of one packed block (fields of mask, width
 *   columns, every row and plane of the box).
 * les_dd_pack / les_dd_unpack: columns i0..i0+width-1 of the fields in
 *   mask (bit LES_F_*) to / from a device buffer, on the context's stream.
 * les_dd_sums: device address of the context's kLimbs = 6 int64: after a
 *   phase that ends in "sum" this rank's total, to be replaced by the sum
 *   over the ranks before the next phase.
 * les_dd_local_sum: that replacement for n ranks of this process on one
 *   device (one kernel on ranks[0]'s stream, ordered by events against
 *   every rank's stream). */
enum {
    LES_DD_BEGIN = 0,
    LES_DD_MOMENTUM = 1,
    LES_DD_RHSAV = 2,
    LES_DD_SOR_ITER = 3,
    LES_DD_SOR_TEST = 4,
    LES_DD_PAV_SUM = 5,
    LES_DD_PAV_END = 6
};
les_status les_dd_area_part(les_ctx *ctx, int olo, int ohi, unsigned long long *lo, long long *hi, int *bad);
les_status les_dd_set_owned(les_ctx *ctx, int olo, int ohi, unsigned long long area_lo, long long area_hi,
                            int area_bad);
long long les_dd_block_floats(les_ctx *ctx, unsigned mask, int width);
les_status les_dd_pack(les_ctx *ctx, unsigned mask, int i0, int width, float *buf);
les_status les_dd_unpack(les_ctx *ctx, unsigned mask, int i0, int width, const float *buf);
les_status les_dd_sums(les_ctx *ctx, long long **dptr);
les_status les_dd_local_sum(int n, les_ctx *const *ranks);
les_status les_dd_phase(les_ctx *ctx, int phase, int arg);

#ifdef __cplusplus
}
#endif
#endif
