/*
 * CPU oracle for the NICAM horizontal tracer-advection path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference arm of bench.py may
 * load it.  The product path (icoatmosbenchmark_v1_b200) never links or calls it.
 *
 * It is a line-faithful C restatement of the reference Fortran kernels
 * (IcoAtmosBenchmark_v1, kernels/NICAM/...), keeping loop orders, halo-zeroing
 * order, index clamps, Fortran SIGN semantics and left-to-right evaluation, so
 * that a build without FP contraction (-ffp-contract=off) reproduces the
 * reference arithmetic operation by operation.
 *
 * Array layout: Fortran column-major var(ij,k,l[,m]) == C row-major
 * var[m][l][k][ij]; pole arrays var_pl(6,k,2[,m]).  Indices i,j,ij inside the
 * restated loops are Fortran 1-based, exactly as in the reference source.
 *
 * Parity status:
 *   horizontal_flux, horizontal_limiter_thuburn, vertical_limiter_thuburn:
 *       restated from the reference; the reference's input snapshots are not
 *       distributed with it, so these are pinned against the restatement only.
 *   COMM list generation / data transfer / COMM_var:
 *       pinned bit-for-bit against the reference's golden logs
 *       kernels/NICAM/communication/reference/msg.pe00000{0,1}.* (gl4 rl0, 2 ranks).
 *   Gradient apply, remap, Courant numbers, rhogq update, vertical flux and
 *   the composed step: not present in the reference; written from the method
 *   description (docs/NICAM/src/20_intro_nicam.tex:368-429) -> parity unpinned,
 *   checked by properties (constancy, monotonicity, conservation).
 */
#ifndef ICOADV_ORACLE_H
#define ICOADV_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sizes of one process' arrays (mod_adm.f90:220-251, problem_size.inc:28-59). */
typedef struct {
  int glevel, rlevel;   /* grid / region division level                        */
  int kall, kmin, kmax; /* vertical grid, Fortran 1-based kmin/kmax            */
  int lall;             /* regular regions held by this process                */
  int have_pl;          /* this process holds the two pole regions             */
  int gall_1d, gall;    /* derived: 2^(gl-rl)+2, gall_1d^2                     */
  int gmin, gmax;       /* derived: 2, gall_1d-1                               */
  int gall_pl, lall_pl; /* 6, 2                                                */
} orc_dims;

void orc_dims_fill(orc_dims *d);

/* ---- A1: horizontal_flux (dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-379) */
void orc_horizontal_flux(const orc_dims *d, const int *have_sgp,
                         double *flx_h, double *flx_h_pl,
                         double *GRD_xc, double *GRD_xc_pl,
                         const double *rho, const double *rho_pl,
                         const double *rhovx, const double *rhovx_pl,
                         const double *rhovy, const double *rhovy_pl,
                         const double *rhovz, const double *rhovz_pl,
                         double dt,
                         const double *GRD_xr, const double *GRD_xr_pl,
                         const double *GMTR_p, const double *GMTR_p_pl,
                         const double *GMTR_t, const double *GMTR_t_pl,
                         const double *GMTR_a, const double *GMTR_a_pl);

/* ---- A2: horizontal_limiter_thuburn (dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-430)
 * Qout_post == NULL selects the original NICAM behaviour: the Qout halo is
 * filled by COMM_data_transfer (single process, list built from `topo`). */
struct orc_topo;
void orc_horizontal_limiter_thuburn(const orc_dims *d, const int *have_sgp,
                                    double *q_a, double *q_a_pl,
                                    const double *q, const double *q_pl,
                                    const double *dd, const double *d_pl,
                                    const double *ch, const double *ch_pl,
                                    const double *cmask, const double *cmask_pl,
                                    double *Qout_prev, double *Qout_prev_pl,
                                    const double *Qout_post, const double *Qout_post_pl,
                                    const struct orc_topo *topo);

/* ---- A3: vertical_limiter_thuburn (dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-243) */
void orc_vertical_limiter_thuburn(const orc_dims *d,
                                  double *q_h, double *q_h_pl,
                                  const double *q, const double *q_pl,
                                  const double *dd, const double *d_pl,
                                  const double *ck, const double *ck_pl);

/* ---- A4: region topology + COMM lists + data transfer (communication/src) */
typedef struct orc_topo orc_topo;
/* Builds mod_adm / mod_comm state for nprocs emulated ranks. */
orc_topo *orc_topo_create(int glevel, int rlevel, int nprocs);
void orc_topo_destroy(orc_topo *t);
int orc_topo_lall(const orc_topo *t);          /* regions per rank          */
int orc_topo_rgn_nmax(const orc_topo *t);
int orc_topo_have_sgp(const orc_topo *t, int rank, int l); /* l 1-based     */
int orc_topo_rgnid(const orc_topo *t, int rank, int l);    /* lp2r          */
void orc_topo_edge_tab(const orc_topo *t, int *out /* [rgn][4][2] */);
void orc_topo_vert_num(const orc_topo *t, int *out /* [rgn][4] */);
int orc_topo_rgn4pl(const orc_topo *t, int pole /* 1 N, 2 S */);
/* var[rank] has shape (gall,kmax,lall,vmax) Fortran order; var_pl[rank]
 * (6,kmax,2,vmax).  Emulates MPI pack / local copy / unpack / singular
 * order of COMM_data_transfer (mod_comm.f90:1506-1891) across all ranks. */
void orc_comm_data_transfer(const orc_topo *t, double **var, double **var_pl,
                            int kmax, int vmax);
/* COMM_var (mod_comm.f90:1895-2101): halo -> pole centre, then data transfer. */
void orc_comm_var(const orc_topo *t, double **var, double **var_pl,
                  int kmax, int vmax);
/* number of rellist entries (COMM_list_generate) of rank 1, for the log check */
int orc_topo_rellist_nmax(const orc_topo *t, int rank);

/* ---- composed step pieces (absent from the reference, parity unpinned) */
void orc_gradient(const orc_dims *d, const int *have_sgp,
                  double *grad, double *grad_pl,              /* (gall,kall,lall,3) */
                  const double *q, const double *q_pl,
                  const double *coef_grad, const double *coef_grad_pl);
void orc_courant(const orc_dims *d, double *ch, double *ch_pl,
                 double *cmask, double *cmask_pl,
                 const double *flx_h, const double *flx_h_pl,
                 const double *rho, const double *rho_pl);
void orc_remap(const orc_dims *d,
               double *q_a, double *q_a_pl,
               const double *q, const double *q_pl,
               const double *grad, const double *grad_pl,
               const double *cmask, const double *cmask_pl,
               const double *GRD_xc, const double *GRD_xc_pl,
               const double *GRD_x, const double *GRD_x_pl);

/* One full tracer step for ntr tracers (see oracle_step.c for the definition).
 * State: rhog (gall,kall,lall) + pole, rhogq (gall,kall,lall,ntr) + pole.
 * Fields (fixed during the step): rhogvx/vy/vz (cell centres),
 * rhogw (half levels, index k = face between k-1 and k).
 * Vertical grid: rdgz (kall), afact/bfact (kall).
 * Halos of rhog and rhogq must be valid on entry and are valid on exit. */
void orc_step(const orc_dims *d, const int *have_sgp, const orc_topo *topo,
              int ntr, double dt,
              double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
              const double *rhogvx, const double *rhogvx_pl,
              const double *rhogvy, const double *rhogvy_pl,
              const double *rhogvz, const double *rhogvz_pl,
              const double *rhogw, const double *rhogw_pl,
              const double *rdgz, const double *afact, const double *bfact,
              const double *GRD_x, const double *GRD_x_pl,
              const double *GRD_xr, const double *GRD_xr_pl,
              const double *GMTR_p, const double *GMTR_p_pl,
              const double *GMTR_t, const double *GMTR_t_pl,
              const double *GMTR_a, const double *GMTR_a_pl,
              const double *coef_grad, const double *coef_grad_pl,
              int nthreads);

/* Adjoint of orc_step (oracle_adjoint.c): given the step's input state and, in
 * a_rhog / a_rhogq (+ _pl), the adjoint of its output, overwrites them with the
 * adjoint of its input and adds the adjoint of rhogvx/vy/vz (+ _pl) to a_vx/a_vy/a_vz. */
void orc_step_adjoint(const orc_dims *d, const int *have_sgp, const orc_topo *topo, int ntr, double dt,
                      const double *rhog, const double *rhog_pl, const double *rhogq, const double *rhogq_pl,
                      const double *rhogvx, const double *rhogvx_pl, const double *rhogvy, const double *rhogvy_pl,
                      const double *rhogvz, const double *rhogvz_pl, const double *rhogw, const double *rhogw_pl,
                      const double *rdgz, const double *afact, const double *bfact,
                      const double *GRD_x, const double *GRD_x_pl, const double *GRD_xr, const double *GRD_xr_pl,
                      const double *GMTR_p, const double *GMTR_p_pl, const double *GMTR_t, const double *GMTR_t_pl,
                      const double *GMTR_a, const double *GMTR_a_pl, const double *coef_grad,
                      const double *coef_grad_pl, double *a_rhog, double *a_rhog_pl, double *a_rhogq,
                      double *a_rhogq_pl, double *a_vx, double *a_vx_pl, double *a_vy, double *a_vy_pl, double *a_vz,
                      double *a_vz_pl);

#ifdef __cplusplus
}
#endif
#endif
