/*
 * icoadv: B200 (sm_100a) implementation of the NICAM horizontal tracer
 * advection path of IcoAtmosBenchmark_v1, behind a C ABI.
 *
 * The kernel entry points keep the argument lists of the reference Fortran
 * subroutines, in the same order and with the same array layouts
 * (Fortran column-major, e.g. flx_h(ADM_gall,ADM_kall,ADM_lall,6) is a
 * contiguous double[6][lall][kall][gall]).  What the reference reads from
 * module globals (ADM_* sizes, CONST_EPS/CONST_HUGE, ADM_have_sgp, GRD_xr and
 * the GMTR_* metrics) is held by the context: sizes are fixed by ica_init and
 * the metrics are registered once with ica_set_geometry.
 *
 * One context covers one whole icosahedral grid on one GPU: all
 * 10*4^rlevel regions (ADM_lall) and both pole regions (ADM_have_pl = true).
 *
 * Host-pointer entry points copy their inputs to the device, run on the
 * context's stream and copy the outputs back before returning.  The *_dev
 * variants take device pointers of the same shapes and are asynchronous on
 * the context's stream (ica_stream).  Every function returns ICA_OK (0) or a
 * negative ICA_ERR_* code; the reference has no status returns (it stops),
 * so a Fortran shim over this header turns a nonzero status into STOP.
 *
 * Precision: the reference selects RP at compile time (mod_precision.f90:19-26);
 * here the unsuffixed entry points are RP = DP (double), the *_f32 ones are
 * RP = SP (float, EPS = epsilon(1.0), HUGE = huge(1.0)).
 */
#ifndef ICOADV_H
#define ICOADV_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ICA_OK 0
#define ICA_ERR_ARG (-1)      /* bad size, NULL pointer or out-of-range argument */
#define ICA_ERR_STATE (-2)    /* context not initialised / geometry not registered */
#define ICA_ERR_CUDA (-3)     /* a CUDA call failed; see ica_last_error() */
#define ICA_ERR_TIMEOUT (-4)  /* a bounded device-side wait gave up */
#define ICA_ERR_INTERNAL (-5) /* an internal consistency check failed */
#define ICA_ERR_NOMEM (-6)    /* device or host allocation failed */

typedef struct ica_ctx ica_ctx;

/* Sizes.  Replaces the ADM_* module globals of problem_size.inc:28-59 and the
 * ADMPARAM namelist of communication/src/mod_adm.f90:172-251:
 * gall_1d = 2^(glevel-rlevel)+2, gmin = 2, gmax = gall_1d-1,
 * lall = 10*4^rlevel, kall = vlayer+2, kmin = 2, kmax = vlayer+1
 * (vlayer = 1 gives kall = kmin = kmax = 1). */
typedef struct {
  int glevel;
  int rlevel;
  int vlayer;
  int device; /* CUDA device ordinal */
} ica_dims;

/* Derived sizes, for callers that allocate arrays. */
typedef struct {
  int gall_1d, gall, gmin, gmax; /* 1-based Fortran indices gmin/gmax */
  int kall, kmin, kmax;
  int lall, gall_pl, lall_pl;    /* lall_pl = 2, gall_pl = 6 */
} ica_sizes;

/* Create a context: sizes, the CUDA stream and the halo/pole gather plan.
 * Replaces ADM_setup + COMM_setup (mod_adm.f90:165, mod_comm.f90:147). */
int ica_init(const ica_dims *dims, ica_ctx **ctx);
/* A context for arrays that hold part of a grid, sized by the module globals the reference's
 * kernel drivers keep (kernels/NICAM/dyn_horiz_adv_flux/src/problem_size.inc:28-50):
 * ADM_gall_1d, ADM_kall, ADM_kmin, ADM_kmax, ADM_lall, ADM_have_pl and
 * ADM_have_sgp(1:ADM_lall) (0 or 1); ADM_gall = gall_1d^2, ADM_gmin = 2,
 * ADM_gmax = gall_1d - 1.  The drivers' own case, one region of a glevel-7 grid and both
 * poles, is (130, 42, 2, 41, 1, 1, {1}).  The kernel entry points (horizontal_flux,
 * horizontal_limiter_thuburn with Qout_post given, vertical_limiter_thuburn) run on such
 * arrays as on a whole grid, and have_pl = 0 leaves the pole arrays untouched, as the
 * reference's `if (ADM_have_pl)` blocks do.  The context holds no region topology, so the
 * COMM entry points, the limiter's on-GPU Qout fill (Qout_post = NULL), the composed steps
 * and the batched path return ICA_ERR_STATE: the neighbours of a region are not known. */
int ica_init_regions(int gall_1d, int kall, int kmin, int kmax, int lall, int have_pl,
                     const int *have_sgp, int device, ica_ctx **ctx);
int ica_finalize(ica_ctx *ctx);
int ica_get_sizes(const ica_ctx *ctx, ica_sizes *out);
/* The context's CUDA stream (a cudaStream_t), for the *_dev entry points. */
void *ica_stream(ica_ctx *ctx);
/* Text of the last error on this thread. */
const char *ica_last_error(void);
/* Number of kernels this library launched since the context was created. */
long long ica_launch_count(const ica_ctx *ctx);
/* Is the library's device code loadable on `device` (sm_100)?  0 = yes. */
int ica_device_check(int device);

/* Metrics read by horizontal_flux from module mod_misc (mod_misc.f90:128-136;
 * dyn_horiz_adv_flux/src/main.f90:91-98 for the shapes):
 *   GRD_xr(gall,1,lall,3,3)  GRD_xr_pl(6,1,2,3)
 *   GMTR_p(gall,1,lall,8)    GMTR_p_pl(6,1,2,8)
 *   GMTR_t(gall,1,lall,2,5)  GMTR_t_pl(6,1,2,5)
 *   GMTR_a(gall,1,lall,3,12) GMTR_a_pl(6,1,2,18)
 * Copied to the device once (FP64, and an FP32 copy for the *_f32 path). */
int ica_set_geometry(ica_ctx *ctx,
                     const double *GRD_xr, const double *GRD_xr_pl,
                     const double *GMTR_p, const double *GMTR_p_pl,
                     const double *GMTR_t, const double *GMTR_t_pl,
                     const double *GMTR_a, const double *GMTR_a_pl);

/* The grid and its metrics built on the device, for a whole-grid context (ica_init): the cell
 * positions of this library's icosahedral grid (recursive bisection of the ten diamonds of the
 * region table, radius `radius`) and from them the setup of the reference's dyn_metrics kernel,
 * GMTR_p/t/a_setup (kernels/NICAM/dyn_metrics/src/mod_gmtr.f90:46-741) and OPRT_gradient_setup
 * (dyn_metrics/src/mod_oprt.f90:499-734), with the halo fills of COMM.  Device arrays, written
 * asynchronously on the context stream, in the layouts ica_set_geometry and
 * ica_set_step_geometry read: GRD_x(gall,1,lall,3) GRD_x_pl(6,1,2,3), GRD_xr(gall,1,lall,3,3)
 * GRD_xr_pl(6,1,2,3), GMTR_p(gall,1,lall,8) GMTR_p_pl(6,1,2,8), GMTR_t(gall,1,lall,2,5)
 * GMTR_t_pl(6,1,2,5), GMTR_a(gall,1,lall,3,12) GMTR_a_pl(6,1,2,18), coef_grad(gall,0:6,3,lall)
 * coef_grad_pl(0:5,3,2).  Context scratch: about 9 doubles per cell. */
int ica_grid_build_dev(ica_ctx *ctx, double radius,
                       double *GRD_x, double *GRD_x_pl, double *GRD_xr, double *GRD_xr_pl,
                       double *GMTR_p, double *GMTR_p_pl, double *GMTR_t, double *GMTR_t_pl,
                       double *GMTR_a, double *GMTR_a_pl, double *coef_grad, double *coef_grad_pl);

/* ---- horizontal_flux: kernels/NICAM/dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-49,78-90
 * out flx_h(gall,kall,lall,6) flx_h_pl(6,kall,2)
 *     GRD_xc(gall,kall,lall,3,3) GRD_xc_pl(6,kall,2,3)
 * in  rho, rhovx, rhovy, rhovz (gall,kall,lall) + _pl (6,kall,2), dt */
int ica_horizontal_flux(ica_ctx *ctx,
                        double *flx_h, double *flx_h_pl,
                        double *GRD_xc, double *GRD_xc_pl,
                        const double *rho, const double *rho_pl,
                        const double *rhovx, const double *rhovx_pl,
                        const double *rhovy, const double *rhovy_pl,
                        const double *rhovz, const double *rhovz_pl,
                        double dt);
int ica_horizontal_flux_dev(ica_ctx *ctx,
                            double *flx_h, double *flx_h_pl,
                            double *GRD_xc, double *GRD_xc_pl,
                            const double *rho, const double *rho_pl,
                            const double *rhovx, const double *rhovx_pl,
                            const double *rhovy, const double *rhovy_pl,
                            const double *rhovz, const double *rhovz_pl,
                            double dt);
int ica_horizontal_flux_f32(ica_ctx *ctx,
                            float *flx_h, float *flx_h_pl,
                            float *GRD_xc, float *GRD_xc_pl,
                            const float *rho, const float *rho_pl,
                            const float *rhovx, const float *rhovx_pl,
                            const float *rhovy, const float *rhovy_pl,
                            const float *rhovz, const float *rhovz_pl,
                            float dt);

/* ---- horizontal_limiter_thuburn:
 *      kernels/NICAM/dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-49,71-84
 * inout q_a(gall,kall,lall,6) q_a_pl(6,kall,2)
 * in    q, d (gall,kall,lall); ch, cmask (gall,kall,lall,6); + _pl (6,kall,2)
 * out   Qout_prev(gall,kall,lall,2) Qout_prev_pl(6,kall,2,2): Qout before the halo fill
 * in    Qout_post(gall,kall,lall,2) Qout_post_pl(6,kall,2,2): Qout after the halo fill,
 *       as the extracted kernel reads it from its snapshot (:369-373).  Pass NULL
 *       for both to run the fill on the GPU instead, which is what NICAM does
 *       (the commented COMM_data_transfer at :371). */
int ica_horizontal_limiter_thuburn(ica_ctx *ctx,
                                   double *q_a, double *q_a_pl,
                                   const double *q, const double *q_pl,
                                   const double *d, const double *d_pl,
                                   const double *ch, const double *ch_pl,
                                   const double *cmask, const double *cmask_pl,
                                   double *Qout_prev, double *Qout_prev_pl,
                                   const double *Qout_post, const double *Qout_post_pl);
int ica_horizontal_limiter_thuburn_dev(ica_ctx *ctx,
                                       double *q_a, double *q_a_pl,
                                       const double *q, const double *q_pl,
                                       const double *d, const double *d_pl,
                                       const double *ch, const double *ch_pl,
                                       const double *cmask, const double *cmask_pl,
                                       double *Qout_prev, double *Qout_prev_pl,
                                       const double *Qout_post, const double *Qout_post_pl);
int ica_horizontal_limiter_thuburn_f32(ica_ctx *ctx,
                                       float *q_a, float *q_a_pl,
                                       const float *q, const float *q_pl,
                                       const float *d, const float *d_pl,
                                       const float *ch, const float *ch_pl,
                                       const float *cmask, const float *cmask_pl,
                                       float *Qout_prev, float *Qout_prev_pl,
                                       const float *Qout_post, const float *Qout_post_pl);

/* ica_horizontal_limiter_thuburn_dev without any device allocation.  No reference
 * counterpart: it serves callers that cannot let a library allocate device memory
 * after start-up (a host model whose pool allocator owns the GPU, a run whose
 * footprint must stay fixed).  The scratch (the Qout copy the halo fill runs on and
 * the pole inflow bounds) is a fixed array in the library's device memory, about
 * 32.1 MiB.  ica_init looks up its address on the context's device, which loads it
 * there, so create the context before a pool allocator claims the GPU; every GPU
 * with a context then holds the array until the process exits.  (Should that lookup
 * fail, the first call repeats it: make that call before any stream capture.)  Grids with
 * gall*kall*lall > ICA_NOALLOC_MAX_CELLS or kall > ICA_NOALLOC_MAX_KALL get
 * ICA_ERR_ARG.  Nothing needs to start at zero.  All calls share the one array, so
 * calls that overlap on a GPU (other streams, other host threads) race. */
#define ICA_NOALLOC_MAX_CELLS 2097152
#define ICA_NOALLOC_MAX_KALL 256
int ica_horizontal_limiter_thuburn_noalloc(ica_ctx *ctx,
                                           double *q_a, double *q_a_pl,
                                           const double *q, const double *q_pl,
                                           const double *d, const double *d_pl,
                                           const double *ch, const double *ch_pl,
                                           const double *cmask, const double *cmask_pl,
                                           double *Qout_prev, double *Qout_prev_pl,
                                           const double *Qout_post, const double *Qout_post_pl);

/* ---- vertical_limiter_thuburn:
 *      kernels/NICAM/dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-45,60-67
 * inout q_h(gall,kall,lall) q_h_pl(6,kall,2)
 * in    q, d (gall,kall,lall) + _pl; ck(gall,kall,lall,2) ck_pl(6,kall,2,2) */
int ica_vertical_limiter_thuburn(ica_ctx *ctx,
                                 double *q_h, double *q_h_pl,
                                 const double *q, const double *q_pl,
                                 const double *d, const double *d_pl,
                                 const double *ck, const double *ck_pl);
int ica_vertical_limiter_thuburn_dev(ica_ctx *ctx,
                                     double *q_h, double *q_h_pl,
                                     const double *q, const double *q_pl,
                                     const double *d, const double *d_pl,
                                     const double *ck, const double *ck_pl);
int ica_vertical_limiter_thuburn_f32(ica_ctx *ctx,
                                     float *q_h, float *q_h_pl,
                                     const float *q, const float *q_pl,
                                     const float *d, const float *d_pl,
                                     const float *ck, const float *ck_pl);

/* ---- COMM_data_transfer: kernels/NICAM/communication/src/mod_comm.f90:1506-1540
 * inout var(gall,kmax,lall,vmax) var_pl(6,kmax,2,vmax).  The reference takes
 * kmax and vmax from shape(var); here they are arguments.  The MPI exchange
 * of the reference becomes one bit-exact index gather on the GPU. */
int ica_comm_data_transfer(ica_ctx *ctx, double *var, double *var_pl, int kmax, int vmax);
int ica_comm_data_transfer_dev(ica_ctx *ctx, double *var, double *var_pl, int kmax, int vmax);
int ica_comm_data_transfer_f32(ica_ctx *ctx, float *var, float *var_pl, int kmax, int vmax);
/* ---- COMM_var: mod_comm.f90:1895-1917 (halo -> pole centre, then the transfer) */
int ica_comm_var(ica_ctx *ctx, double *var, double *var_pl, int kmax, int vmax);
int ica_comm_var_dev(ica_ctx *ctx, double *var, double *var_pl, int kmax, int vmax);

/* ---- The composed tracer step (not in the reference, which runs each kernel
 * alone on a snapshot).  One step = horizontal_flux -> Courant numbers and
 * upwind masks -> gradient (OPRT_gradient_setup stencil, dyn_metrics/src/
 * mod_oprt.f90:499-734) + halo fill -> Miura upwind remap -> Thuburn horizontal
 * limiter with the Qout halo fill -> rhogq/rhog update, then the vertical
 * sub-step (vertical_limiter_thuburn on linearly interpolated half-level
 * values) and the halo fill of the state.
 *
 * Step geometry: cell positions GRD_x(gall,1,lall,3) GRD_x_pl(6,1,2,3);
 * coef_grad(gall,0:6,3,lall) coef_grad_pl(0:5,3,2); vertical grid rdgz(kall),
 * afact(kall), bfact(kall) with q_h(k) = afact(k) q(k) + bfact(k) q(k-1) at
 * the face between levels k-1 and k. */
int ica_set_step_geometry(ica_ctx *ctx, const double *GRD_x, const double *GRD_x_pl,
                          const double *coef_grad, const double *coef_grad_pl,
                          const double *rdgz, const double *afact, const double *bfact);
/* Plain FP64 step, tracer by tracer.  State (in/out, halos valid on entry and
 * exit): rhog(gall,kall,lall) rhog_pl(6,kall,2), rhogq(gall,kall,lall,ntr)
 * rhogq_pl(6,kall,2,ntr).  Fields: rhogvx/vy/vz(gall,kall,lall) + _pl at cell
 * centres, rhogw(gall,kall,lall) + _pl at the face below each level (zero at
 * the ground face kmin and the top face kmax+1). */
int ica_advect_step(ica_ctx *ctx, int ntr, double dt,
                    double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                    const double *rhogvx, const double *rhogvx_pl,
                    const double *rhogvy, const double *rhogvy_pl,
                    const double *rhogvz, const double *rhogvz_pl,
                    const double *rhogw, const double *rhogw_pl);
int ica_advect_step_dev(ica_ctx *ctx, int ntr, double dt,
                        double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                        const double *rhogvx, const double *rhogvx_pl,
                        const double *rhogvy, const double *rhogvy_pl,
                        const double *rhogvz, const double *rhogvz_pl,
                        const double *rhogw, const double *rhogw_pl);

/* Adjoint (reverse mode) of the plain FP64 step, for gradients of a function
 * of the state after the step.  Subgradients at the limiter kinks: min / max /
 * clamp pass the adjoint to the operand the forward step returned, the upwind
 * masks, inflow flags and zero-outflow switches are held fixed, and the
 * +-BIG terms of a masked bound carry no derivative.  rhogw, the geometry and
 * the vertical grid are constants.
 *   in:      the step's input state (rhog, rhogq + pole arrays; unchanged), the fields
 *   in/out:  a_rhog(gall,kall,lall) a_rhog_pl, a_rhogq(gall,kall,lall,ntr) a_rhogq_pl:
 *            the adjoint of the step's output on entry, of its input on return
 *   +=:      a_rhogvx/vy/vz (+ _pl), the adjoint of the horizontal wind
 * Needs 4 <= kall <= 128.  Halo points of the adjoint follow the state's halo
 * fill: on return the adjoint of a halo point is what the step's output depends
 * on it through (its own value before the fill), not a copy. */
int ica_advect_step_adjoint_dev(ica_ctx *ctx, int ntr, double dt,
                                const double *rhog, const double *rhog_pl,
                                const double *rhogq, const double *rhogq_pl,
                                const double *rhogvx, const double *rhogvx_pl,
                                const double *rhogvy, const double *rhogvy_pl,
                                const double *rhogvz, const double *rhogvz_pl,
                                const double *rhogw, const double *rhogw_pl,
                                double *a_rhog, double *a_rhog_pl,
                                double *a_rhogq, double *a_rhogq_pl,
                                double *a_rhogvx, double *a_rhogvx_pl,
                                double *a_rhogvy, double *a_rhogvy_pl,
                                double *a_rhogvz, double *a_rhogvz_pl);
int ica_advect_step_adjoint(ica_ctx *ctx, int ntr, double dt,
                            const double *rhog, const double *rhog_pl,
                            const double *rhogq, const double *rhogq_pl,
                            const double *rhogvx, const double *rhogvx_pl,
                            const double *rhogvy, const double *rhogvy_pl,
                            const double *rhogvz, const double *rhogvz_pl,
                            const double *rhogw, const double *rhogw_pl,
                            double *a_rhog, double *a_rhog_pl,
                            double *a_rhogq, double *a_rhogq_pl,
                            double *a_rhogvx, double *a_rhogvx_pl,
                            double *a_rhogvy, double *a_rhogvy_pl,
                            double *a_rhogvz, double *a_rhogvz_pl);
/* Multi-step runs with step checkpointing (device pointers, context stream).
 * ica_adjoint_record advances the state nsteps plain FP64 steps in place and
 * keeps a copy of the state every `every` steps (ceil(nsteps/every) states of
 * device memory held by the context).  ica_adjoint_sweep runs the adjoint
 * backwards over the recorded run: each segment is recomputed from its
 * checkpoint (every-1 more states held) and transposed step by step; the
 * a_* arguments mean what they mean for ica_advect_step_adjoint_dev, for the
 * whole run.  The fields must be the ones the run was recorded with.
 * ica_adjoint_release frees the checkpoints and the adjoint scratch. */
int ica_adjoint_record(ica_ctx *ctx, int ntr, double dt, int nsteps, int every,
                       double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                       const double *rhogvx, const double *rhogvx_pl,
                       const double *rhogvy, const double *rhogvy_pl,
                       const double *rhogvz, const double *rhogvz_pl,
                       const double *rhogw, const double *rhogw_pl);
int ica_adjoint_sweep(ica_ctx *ctx,
                      const double *rhogvx, const double *rhogvx_pl,
                      const double *rhogvy, const double *rhogvy_pl,
                      const double *rhogvz, const double *rhogvz_pl,
                      const double *rhogw, const double *rhogw_pl,
                      double *a_rhog, double *a_rhog_pl,
                      double *a_rhogq, double *a_rhogq_pl,
                      double *a_rhogvx, double *a_rhogvx_pl,
                      double *a_rhogvy, double *a_rhogvy_pl,
                      double *a_rhogvz, double *a_rhogvz_pl);
int ica_adjoint_release(ica_ctx *ctx);

/* Batched step: all tracers of the step together, a horizontal kernel (one
 * CTA per region tile and level) and a vertical kernel (one thread per column
 * and tracer); FP32 flux-form remap / limiter arithmetic on interior faces,
 * FP64 on the faces between a region and its halo, FP64 rhog / rhogq update
 * (conservative to FP64 rounding).  Same composition and state layout as ica_advect_step; the
 * fields are FP32.  Device pointers, asynchronous on the context stream; the
 * state goes from the *_in to the *_out buffers (which must differ) with the
 * halos of the output filled.  Needs 4 <= kall <= 128. */
int ica_advect_fast_dev(ica_ctx *ctx, int ntr, double dt,
                        const double *rhog_in, const double *rhog_in_pl,
                        const double *rhogq_in, const double *rhogq_in_pl,
                        double *rhog_out, double *rhog_out_pl,
                        double *rhogq_out, double *rhogq_out_pl,
                        const float *rhogvx, const float *rhogvx_pl,
                        const float *rhogvy, const float *rhogvy_pl,
                        const float *rhogvz, const float *rhogvz_pl,
                        const float *rhogw, const float *rhogw_pl);
/* The same step on host arrays, in place on the state (copies in and out).  The state
 * moves in chunks of tracers on two copy streams, overlapped with the step on the chunk
 * before; from page-locked host memory the copies in and out run at the same time. */
int ica_advect_fast(ica_ctx *ctx, int ntr, double dt,
                    double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                    const float *rhogvx, const float *rhogvx_pl,
                    const float *rhogvy, const float *rhogvy_pl,
                    const float *rhogvz, const float *rhogvz_pl,
                    const float *rhogw, const float *rhogw_pl);
/* ---- Region sharding of the batched step over ranks (one process and GPU per rank).  Every
 * rank holds the whole grid's arrays and computes a contiguous block of regions [l0, l1) (the
 * reference's region order, mod_adm.f90:791-801), rank 0 also the two pole centres
 * (mod_adm.f90:190).  Within a step one region reads another's values in two places, and
 * each becomes an exchange: the boundary values (gradient and Qout of the cells other
 * regions' halos copy, 5 values per tracer and level) after the boundary pass, and the halo
 * fill of the new state.  The caller moves the packed buffers between ranks (NCCL send/recv
 * through torch.distributed in icoatmosbenchmark_v1_b200/shard.py); nothing reads another
 * GPU's memory.
 * ica_shard_set: this context computes regions [l0, l1) (0-based) and, if poles, the pole
 * centres; dst/src[nlocal] (host arrays, points numbered as in ica_comm_plan) are the halo
 * copies whose two points it owns.  nlocal < 0 returns the context to the whole grid.
 * ica_advect_fast_part_dev: part 1 runs the boundary pass, part 2 the rest of the step and
 * the local halo copies; arguments as ica_advect_fast_dev. */
int ica_shard_set(ica_ctx *ctx, int l0, int l1, int poles, int nlocal, const int *dst, const int *src);
int ica_advect_fast_part_dev(ica_ctx *ctx, int part, int ntr, double dt,
                             const double *rhog_in, const double *rhog_in_pl,
                             const double *rhogq_in, const double *rhogq_in_pl,
                             double *rhog_out, double *rhog_out_pl,
                             double *rhogq_out, double *rhogq_out_pl,
                             const float *rhogvx, const float *rhogvx_pl,
                             const float *rhogvy, const float *rhogvy_pl,
                             const float *rhogvz, const float *rhogvz_pl,
                             const float *rhogw, const float *rhogw_pl);
/* Pack / unpack, device pointers, context stream: the boundary values of the boundary indices
 * bidx[n] (as ica_boundary_tables numbers them) between the context's boundary buffer and
 * buf(5, n, kall, ntr); the points pts[n] of var(gall,kmax,lall,vmax) + var_pl(6,kmax,2,vmax)
 * and buf(n, kmax, vmax). */
int ica_shard_bval_pack(ica_ctx *ctx, int ntr, int n, const int *bidx, double *buf);
int ica_shard_bval_unpack(ica_ctx *ctx, int ntr, int n, const int *bidx, const double *buf);
int ica_shard_points_pack(ica_ctx *ctx, int n, const int *pts, int kmax, int vmax,
                          const double *var, const double *var_pl, double *buf);
int ica_shard_points_unpack(ica_ctx *ctx, int n, const int *pts, int kmax, int vmax,
                            double *var, double *var_pl, const double *buf);
/* FP64 variant of the batched step: the same kernels with every face value, bound,
 * Courant number and limiter in FP64 and FP64 fields, so the result follows the plain
 * FP64 step to FP64 rounding (the FP32 variant differs from it at FP32 rounding). */
int ica_advect_fast64_dev(ica_ctx *ctx, int ntr, double dt,
                          const double *rhog_in, const double *rhog_in_pl,
                          const double *rhogq_in, const double *rhogq_in_pl,
                          double *rhog_out, double *rhog_out_pl,
                          double *rhogq_out, double *rhogq_out_pl,
                          const double *rhogvx, const double *rhogvx_pl,
                          const double *rhogvy, const double *rhogvy_pl,
                          const double *rhogvz, const double *rhogvz_pl,
                          const double *rhogw, const double *rhogw_pl);
/* Tile shapes of the horizontal kernel (TX x TY cells, TG tracers per batch): *n shapes;
 * tx/ty/tg (may be NULL) receive them.  ica_fast_set_shape selects one (the
 * autotuner in the Python layer times them and keeps the fastest). */
int ica_fast_shapes(ica_ctx *ctx, int *n, int *tx, int *ty, int *tg);
int ica_fast_set_shape(ica_ctx *ctx, int shape);
/* Tracers per chunk of ica_advect_fast's copies; 0 (the default) sizes chunks at about
 * 1 GiB of rhogq, 1 to 4 tracers.  The result does not depend on it. */
int ica_fast_set_host_chunk(ica_ctx *ctx, int tracers);
/* Status of the batched kernels since the last call: *flags = 0, or bit 0 set if a wait of the
 * horizontal kernel for its tile copies (TMA) gave up after its time limit (the step's result
 * is then invalid); returns ICA_ERR_TIMEOUT in that case.  Synchronises the stream and clears
 * the flags. */
int ica_fast_status(ica_ctx *ctx, int *flags);
/* CUDA-event timing of the horizontal kernel: returns the total milliseconds and
 * the number of launches recorded since the last call, then enables (1) or
 * disables (0) recording for the following calls.  Synchronises the stream. */
int ica_fast_timing(ica_ctx *ctx, int enable, double *ms_total, long long *count);

/* ---- Batches: up to ICA_BATCH_MAX grid instances (for example uneven grid levels, each
 * with its own context, geometry and tracer count) advanced by the same launches: every
 * stage of ica_advect_fast_dev is one launch over the work of all instances, the horizontal
 * kernel persistent (one wave of CTAs striding over (instance, level, tile) items).  The
 * work runs on the first context's stream.  A step can be captured into a CUDA graph
 * (two slots, for the two directions of a double-buffered state) and replayed; capture
 * only after one uncaptured ica_batch_step_dev with the same arguments has set up every
 * instance's device buffers.  Instances must live on the same device. */
#define ICA_BATCH_MAX 4
typedef struct ica_batch ica_batch;
typedef struct {
  int ntr;
  double dt;
  const double *rhog_in, *rhog_in_pl, *rhogq_in, *rhogq_in_pl;
  double *rhog_out, *rhog_out_pl, *rhogq_out, *rhogq_out_pl;
  const float *rhogvx, *rhogvx_pl, *rhogvy, *rhogvy_pl, *rhogvz, *rhogvz_pl, *rhogw, *rhogw_pl;
} ica_fast_args;
int ica_batch_create(ica_ctx *const *ctxs, int n, ica_batch **out);
int ica_batch_destroy(ica_batch *b);
/* Tile shape (index into ica_fast_shapes) used for every instance of the batch. */
int ica_batch_set_shape(ica_batch *b, int shape);
/* One step of every instance (args[i] for instance i), device pointers, asynchronous. */
int ica_batch_step_dev(ica_batch *b, const ica_fast_args *args);
/* The FP64 variant of a batch: FP64 fields (ica_fast_args64); all instances of a step
 * use one variant. */
typedef struct {
  int ntr;
  double dt;
  const double *rhog_in, *rhog_in_pl, *rhogq_in, *rhogq_in_pl;
  double *rhog_out, *rhog_out_pl, *rhogq_out, *rhogq_out_pl;
  const double *rhogvx, *rhogvx_pl, *rhogvy, *rhogvy_pl, *rhogvz, *rhogvz_pl, *rhogw, *rhogw_pl;
} ica_fast_args64;
int ica_batch_step64_dev(ica_batch *b, const ica_fast_args64 *args);
/* Capture the step with these arguments into graph slot 0 or 1 (replacing what was there). */
int ica_batch_capture(ica_batch *b, const ica_fast_args *args, int slot);
int ica_batch_capture64(ica_batch *b, const ica_fast_args64 *args, int slot);
/* Launch the graph in slot 0 or 1 on the batch stream. */
int ica_batch_replay(ica_batch *b, int slot);

/* ---- Host-only topology helpers (no GPU needed).
 * Point index of region cell (i,j) of region r (all 1-based):
 *   (r-1)*gall + (j-1)*gall_1d + (i-1);  pole p (0 north, 1 south), slot v:
 *   10*4^rlevel*gall + 6*p + (v-1).
 * ica_comm_plan: the composed single-process halo fill dst[e] <- src[e]
 * (pole_fill = 1 adds COMM_var's halo -> pole-centre copy first).  Call with
 * dst = src = NULL to get the count in *n. */
int ica_comm_plan(int glevel, int rlevel, int pole_fill, int *n, int *dst, int *src);
/* have_sgp[10*4^rl] (ADM_have_sgp), rgn4pl[2] (RGNMNG_rgn4pl),
 * pole_ring[2][5] (RGNMNG_vert_tab_pl region ids); any may be NULL. */
int ica_topology_info(int glevel, int rlevel, int *have_sgp, int *rgn4pl, int *pole_ring);
/* ica_boundary_tables (host only): the batched step's boundary-value tables.  bsrc[lall*gall]:
 * a region point's boundary index (a region-boundary cell's own, a halo point's source's;
 * -1 an interior cell off the region boundary, -2 a halo point no list writes); blist[*nb]:
 * the point of each boundary index (region points l*gall + ij, then the two pole centres as
 * lall*gall + 6*p); pole_ring[2][5]: the boundary index feeding each pole ring slot.  Call
 * with NULL arrays to get *nb. */
int ica_boundary_tables(int glevel, int rlevel, int *nb, int *bsrc, int *blist, int *pole_ring);

#ifdef __cplusplus
}
#endif
#endif /* ICOADV_H */
