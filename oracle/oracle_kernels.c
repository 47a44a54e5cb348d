/*
 * CPU oracle: line-faithful restatement of the three reference tracer kernels.
 * TEST INFRASTRUCTURE ONLY (see icoadv_oracle.h).
 *
 *   horizontal_flux            kernels/NICAM/dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-379
 *   horizontal_limiter_thuburn kernels/NICAM/dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-430
 *   vertical_limiter_thuburn   kernels/NICAM/dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-243
 *
 * Loop bounds, statement order and operand order follow the Fortran source so
 * that, compiled with -ffp-contract=off, every value is produced by the same
 * sequence of IEEE operations.  EPS and HUGE are epsilon(1.0d0) and huge(1.0d0)
 * as set by CONST_setup (mod_misc.f90:447-461).
 */
#include "icoadv_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TI 1
#define TJ 2
#define AI 1
#define AIJ 2
#define AJ 3
#define W1 3
#define W2 4
#define W3 5
#define HNX 1
#define HNY 2
#define HNZ 3
#define P_RAREA 2
#define I_min 1
#define I_max 2

/* Fortran MIN/MAX of two reals; written as a comparison so the CUDA kernels
 * can use the identical rule. */
static inline double fmin2(double a, double b) { return (b < a) ? b : a; }
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }
/* Fortran SIGN(a,b) with IEEE signed zero (gfortran: sign(0.5,-0.0) = -0.5) */
static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

void orc_dims_fill(orc_dims *d) {
  int nmax = 1 << (d->glevel - d->rlevel);
  d->gall_1d = nmax + 2;
  d->gall = d->gall_1d * d->gall_1d;
  d->gmin = 2;
  d->gmax = nmax + 1;
  d->gall_pl = 6;
  d->lall_pl = 2;
}

/* index helpers, Fortran 1-based arguments */
#define R3(a, ij, k, l) a[((size_t)((l)-1) * kall + ((k)-1)) * gall + ((ij)-1)]
#define R4(a, ij, k, l, m) a[(((size_t)((m)-1) * lall + ((l)-1)) * kall + ((k)-1)) * gall + ((ij)-1)]
#define R5(a, ij, k, l, m, n) \
  a[((((size_t)((n)-1) * 3 + ((m)-1)) * lall + ((l)-1)) * kall + ((k)-1)) * gall + ((ij)-1)]
#define P3(a, v, k, l) a[((size_t)((l)-1) * kall + ((k)-1)) * gall_pl + ((v)-1)]
#define P4(a, v, k, l, m) a[(((size_t)((m)-1) * lall_pl + ((l)-1)) * kall + ((k)-1)) * gall_pl + ((v)-1)]
/* geometry: (gall,K0=1,lall,...) */
#define GXR(ij, l, a, x) GRD_xr[((((size_t)((x)-1) * 3 + ((a)-1)) * lall + ((l)-1))) * gall + ((ij)-1)]
#define GXR_PL(v, l, x) GRD_xr_pl[(((size_t)((x)-1) * lall_pl + ((l)-1))) * gall_pl + ((v)-1)]
#define GP(ij, l, p) GMTR_p[(((size_t)((p)-1) * lall + ((l)-1))) * gall + ((ij)-1)]
#define GP_PL(v, l, p) GMTR_p_pl[(((size_t)((p)-1) * lall_pl + ((l)-1))) * gall_pl + ((v)-1)]
#define GT(ij, l, t, w) GMTR_t[((((size_t)((w)-1) * 2 + ((t)-1)) * lall + ((l)-1))) * gall + ((ij)-1)]
#define GT_PL(v, l, w) GMTR_t_pl[(((size_t)((w)-1) * lall_pl + ((l)-1))) * gall_pl + ((v)-1)]
#define GA(ij, l, a, h) GMTR_a[((((size_t)((h)-1) * 3 + ((a)-1)) * lall + ((l)-1))) * gall + ((ij)-1)]
#define GA_PL(v, l, h) GMTR_a_pl[(((size_t)((h)-1) * lall_pl + ((l)-1))) * gall_pl + ((v)-1)]

/* ------------------------------------------------------------------------- */
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
                         const double *GMTR_a, const double *GMTR_a_pl) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int gmin = d->gmin, gmax = d->gmax, iall = d->gall_1d;
  const double EPS = DBL_EPSILON;
  double *rhot_TI = calloc(gall, sizeof(double));
  double *rhot_TJ = calloc(gall, sizeof(double));
  double *rhovxt_TI = calloc(gall, sizeof(double));
  double *rhovxt_TJ = calloc(gall, sizeof(double));
  double *rhovyt_TI = calloc(gall, sizeof(double));
  double *rhovyt_TJ = calloc(gall, sizeof(double));
  double *rhovzt_TI = calloc(gall, sizeof(double));
  double *rhovzt_TJ = calloc(gall, sizeof(double));
#define A1(x, ij) x[(ij)-1]
  for (int l = 1; l <= lall; ++l) {
    for (int k = 1; k <= kall; ++k) {
      /* (i,j),(i+1,j)   :141-160 */
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ip1j = ij + 1;
          A1(rhot_TI, ij) = R3(rho, ij, k, l) * GT(ij, l, TI, W1) + R3(rho, ip1j, k, l) * GT(ij, l, TI, W2);
          A1(rhovxt_TI, ij) = R3(rhovx, ij, k, l) * GT(ij, l, TI, W1) + R3(rhovx, ip1j, k, l) * GT(ij, l, TI, W2);
          A1(rhovyt_TI, ij) = R3(rhovy, ij, k, l) * GT(ij, l, TI, W1) + R3(rhovy, ip1j, k, l) * GT(ij, l, TI, W2);
          A1(rhovzt_TI, ij) = R3(rhovz, ij, k, l) * GT(ij, l, TI, W1) + R3(rhovz, ip1j, k, l) * GT(ij, l, TI, W2);
          A1(rhot_TJ, ij) = R3(rho, ij, k, l) * GT(ij, l, TJ, W1);
          A1(rhovxt_TJ, ij) = R3(rhovx, ij, k, l) * GT(ij, l, TJ, W1);
          A1(rhovyt_TJ, ij) = R3(rhovy, ij, k, l) * GT(ij, l, TJ, W1);
          A1(rhovzt_TJ, ij) = R3(rhovz, ij, k, l) * GT(ij, l, TJ, W1);
        }
      /* (i,j+1),(i+1,j+1)   :165-185 */
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ijp1 = ij + iall, ip1jp1 = ij + iall + 1;
          A1(rhot_TI, ij) = A1(rhot_TI, ij) + R3(rho, ip1jp1, k, l) * GT(ij, l, TI, W3);
          A1(rhovxt_TI, ij) = A1(rhovxt_TI, ij) + R3(rhovx, ip1jp1, k, l) * GT(ij, l, TI, W3);
          A1(rhovyt_TI, ij) = A1(rhovyt_TI, ij) + R3(rhovy, ip1jp1, k, l) * GT(ij, l, TI, W3);
          A1(rhovzt_TI, ij) = A1(rhovzt_TI, ij) + R3(rhovz, ip1jp1, k, l) * GT(ij, l, TI, W3);
          A1(rhot_TJ, ij) = A1(rhot_TJ, ij) + R3(rho, ip1jp1, k, l) * GT(ij, l, TJ, W2) + R3(rho, ijp1, k, l) * GT(ij, l, TJ, W3);
          A1(rhovxt_TJ, ij) = A1(rhovxt_TJ, ij) + R3(rhovx, ip1jp1, k, l) * GT(ij, l, TJ, W2) + R3(rhovx, ijp1, k, l) * GT(ij, l, TJ, W3);
          A1(rhovyt_TJ, ij) = A1(rhovyt_TJ, ij) + R3(rhovy, ip1jp1, k, l) * GT(ij, l, TJ, W2) + R3(rhovy, ijp1, k, l) * GT(ij, l, TJ, W3);
          A1(rhovzt_TJ, ij) = A1(rhovzt_TJ, ij) + R3(rhovz, ip1jp1, k, l) * GT(ij, l, TJ, W2) + R3(rhovz, ijp1, k, l) * GT(ij, l, TJ, W3);
        }
      /* singular point   :188-201 */
      if (have_sgp[l - 1]) {
        int j = gmin - 1, i = gmin - 1;
        int ij = (j - 1) * iall + i, ip1j = ij + 1;
        A1(rhot_TI, ij) = A1(rhot_TJ, ip1j);
        A1(rhovxt_TI, ij) = A1(rhovxt_TJ, ip1j);
        A1(rhovyt_TI, ij) = A1(rhovyt_TJ, ip1j);
        A1(rhovzt_TI, ij) = A1(rhovzt_TJ, ip1j);
      }
      /* zero the halo ring   :207-232 */
      for (int j = 1; j <= iall; ++j)
        for (int i = 1; i <= iall; ++i)
          if (i < gmin || i > gmax || j < gmin || j > gmax) {
            int ij = (j - 1) * iall + i;
            for (int m = 1; m <= 6; ++m) R4(flx_h, ij, k, l, m) = 0.0;
            for (int x = 1; x <= 3; ++x)
              for (int a = AI; a <= AJ; ++a) R5(GRD_xc, ij, k, l, a, x) = 0.0;
          }
      /* AI face   :235-257 */
      for (int j = gmin; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ip1j = ij + 1, ijm1 = ij - iall;
          double rrhoa2 = 1.0 / fmax2(A1(rhot_TJ, ijm1) + A1(rhot_TI, ij), EPS);
          double rhovxt2 = A1(rhovxt_TJ, ijm1) + A1(rhovxt_TI, ij);
          double rhovyt2 = A1(rhovyt_TJ, ijm1) + A1(rhovyt_TI, ij);
          double rhovzt2 = A1(rhovzt_TJ, ijm1) + A1(rhovzt_TI, ij);
          double flux = 0.5 * (rhovxt2 * GA(ij, l, AI, HNX) + rhovyt2 * GA(ij, l, AI, HNY) + rhovzt2 * GA(ij, l, AI, HNZ));
          R4(flx_h, ij, k, l, 1) = flux * GP(ij, l, P_RAREA) * dt;
          R4(flx_h, ip1j, k, l, 4) = -flux * GP(ip1j, l, P_RAREA) * dt;
          R5(GRD_xc, ij, k, l, AI, 1) = GXR(ij, l, AI, 1) - rhovxt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AI, 2) = GXR(ij, l, AI, 2) - rhovyt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AI, 3) = GXR(ij, l, AI, 3) - rhovzt2 * rrhoa2 * dt * 0.5;
        }
      /* AIJ face   :261-283 */
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ip1jp1 = ij + iall + 1;
          double rrhoa2 = 1.0 / fmax2(A1(rhot_TI, ij) + A1(rhot_TJ, ij), EPS);
          double rhovxt2 = A1(rhovxt_TI, ij) + A1(rhovxt_TJ, ij);
          double rhovyt2 = A1(rhovyt_TI, ij) + A1(rhovyt_TJ, ij);
          double rhovzt2 = A1(rhovzt_TI, ij) + A1(rhovzt_TJ, ij);
          double flux = 0.5 * (rhovxt2 * GA(ij, l, AIJ, HNX) + rhovyt2 * GA(ij, l, AIJ, HNY) + rhovzt2 * GA(ij, l, AIJ, HNZ));
          R4(flx_h, ij, k, l, 2) = flux * GP(ij, l, P_RAREA) * dt;
          R4(flx_h, ip1jp1, k, l, 5) = -flux * GP(ip1jp1, l, P_RAREA) * dt;
          R5(GRD_xc, ij, k, l, AIJ, 1) = GXR(ij, l, AIJ, 1) - rhovxt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AIJ, 2) = GXR(ij, l, AIJ, 2) - rhovyt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AIJ, 3) = GXR(ij, l, AIJ, 3) - rhovzt2 * rrhoa2 * dt * 0.5;
        }
      /* AJ face   :286-309 */
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ijp1 = ij + iall, im1j = ij - 1;
          double rrhoa2 = 1.0 / fmax2(A1(rhot_TJ, ij) + A1(rhot_TI, im1j), EPS);
          double rhovxt2 = A1(rhovxt_TJ, ij) + A1(rhovxt_TI, im1j);
          double rhovyt2 = A1(rhovyt_TJ, ij) + A1(rhovyt_TI, im1j);
          double rhovzt2 = A1(rhovzt_TJ, ij) + A1(rhovzt_TI, im1j);
          double flux = 0.5 * (rhovxt2 * GA(ij, l, AJ, HNX) + rhovyt2 * GA(ij, l, AJ, HNY) + rhovzt2 * GA(ij, l, AJ, HNZ));
          R4(flx_h, ij, k, l, 3) = flux * GP(ij, l, P_RAREA) * dt;
          R4(flx_h, ijp1, k, l, 6) = -flux * GP(ijp1, l, P_RAREA) * dt;
          R5(GRD_xc, ij, k, l, AJ, 1) = GXR(ij, l, AJ, 1) - rhovxt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AJ, 2) = GXR(ij, l, AJ, 2) - rhovyt2 * rrhoa2 * dt * 0.5;
          R5(GRD_xc, ij, k, l, AJ, 3) = GXR(ij, l, AJ, 3) - rhovzt2 * rrhoa2 * dt * 0.5;
        }
      /* singular point   :311-320 */
      if (have_sgp[l - 1]) {
        int ij = (gmin - 1) * iall + gmin;
        R4(flx_h, ij, k, l, 6) = 0.0;
      }
    }
  }
  /* poles   :326-374 */
  if (d->have_pl) {
    const int n = 1, gmin_pl = 2, gmax_pl = 6;
    double rhot_pl[7], rhovxt_pl[7], rhovyt_pl[7], rhovzt_pl[7];
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k) {
        for (int v = gmin_pl; v <= gmax_pl; ++v) {
          int ij = v, ijp1 = v + 1;
          if (ijp1 == gmax_pl + 1) ijp1 = gmin_pl;
          rhot_pl[v] = P3(rho_pl, n, k, l) * GT_PL(ij, l, W1) + P3(rho_pl, ij, k, l) * GT_PL(ij, l, W2) + P3(rho_pl, ijp1, k, l) * GT_PL(ij, l, W3);
          rhovxt_pl[v] = P3(rhovx_pl, n, k, l) * GT_PL(ij, l, W1) + P3(rhovx_pl, ij, k, l) * GT_PL(ij, l, W2) + P3(rhovx_pl, ijp1, k, l) * GT_PL(ij, l, W3);
          rhovyt_pl[v] = P3(rhovy_pl, n, k, l) * GT_PL(ij, l, W1) + P3(rhovy_pl, ij, k, l) * GT_PL(ij, l, W2) + P3(rhovy_pl, ijp1, k, l) * GT_PL(ij, l, W3);
          rhovzt_pl[v] = P3(rhovz_pl, n, k, l) * GT_PL(ij, l, W1) + P3(rhovz_pl, ij, k, l) * GT_PL(ij, l, W2) + P3(rhovz_pl, ijp1, k, l) * GT_PL(ij, l, W3);
        }
        for (int v = gmin_pl; v <= gmax_pl; ++v) {
          int ij = v, ijm1 = v - 1;
          if (ijm1 == gmin_pl - 1) ijm1 = gmax_pl;
          double rrhoa2 = 1.0 / fmax2(rhot_pl[ijm1] + rhot_pl[ij], EPS);
          double rhovxt2 = rhovxt_pl[ijm1] + rhovxt_pl[ij];
          double rhovyt2 = rhovyt_pl[ijm1] + rhovyt_pl[ij];
          double rhovzt2 = rhovzt_pl[ijm1] + rhovzt_pl[ij];
          double flux = 0.5 * (rhovxt2 * GA_PL(ij, l, HNX) + rhovyt2 * GA_PL(ij, l, HNY) + rhovzt2 * GA_PL(ij, l, HNZ));
          P3(flx_h_pl, v, k, l) = flux * GP_PL(n, l, P_RAREA) * dt;
          P4(GRD_xc_pl, v, k, l, 1) = GXR_PL(v, l, 1) - rhovxt2 * rrhoa2 * dt * 0.5;
          P4(GRD_xc_pl, v, k, l, 2) = GXR_PL(v, l, 2) - rhovyt2 * rrhoa2 * dt * 0.5;
          P4(GRD_xc_pl, v, k, l, 3) = GXR_PL(v, l, 3) - rhovzt2 * rrhoa2 * dt * 0.5;
        }
      }
  }
  free(rhot_TI); free(rhot_TJ); free(rhovxt_TI); free(rhovxt_TJ);
  free(rhovyt_TI); free(rhovyt_TJ); free(rhovzt_TI); free(rhovzt_TJ);
#undef A1
}

/* ------------------------------------------------------------------------- */
void orc_comm_single(const orc_topo *t, double *var, double *var_pl, int kmax, int vmax);

/* Qin(gall,kall,lall,2,6) */
#define QIN(ij, k, l, mm, f) Qin[((((size_t)((f)-1) * 2 + ((mm)-1)) * lall + ((l)-1)) * kall + ((k)-1)) * gall + ((ij)-1)]
#define QIN_PL(v, k, l, mm, f) Qin_pl[((((size_t)((f)-1) * 2 + ((mm)-1)) * lall_pl + ((l)-1)) * kall + ((k)-1)) * gall_pl + ((v)-1)]

void orc_horizontal_limiter_thuburn(const orc_dims *d, const int *have_sgp,
                                    double *q_a, double *q_a_pl,
                                    const double *q, const double *q_pl,
                                    const double *dd, const double *d_pl,
                                    const double *ch, const double *ch_pl,
                                    const double *cmask, const double *cmask_pl,
                                    double *Qout_prev, double *Qout_prev_pl,
                                    const double *Qout_post, const double *Qout_post_pl,
                                    const struct orc_topo *topo) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int gmin = d->gmin, gmax = d->gmax, iall = d->gall_1d;
  const double EPS = DBL_EPSILON, BIG = DBL_MAX;
  /* local work arrays; Qin is never read where the reference leaves it unset */
  double *Qin = calloc((size_t)gall * kall * lall * 12, sizeof(double));
  double *Qin_pl = calloc((size_t)gall_pl * kall * lall_pl * 4, sizeof(double));
  double *Qout = calloc((size_t)gall * kall * lall * 2, sizeof(double));
  double *Qout_pl = calloc((size_t)gall_pl * kall * lall_pl * 2, sizeof(double));

  for (int l = 1; l <= lall; ++l) {
    for (int k = 1; k <= kall; ++k) {
      /* (i) inflow bounds   :143-190 */
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ip1j = ij + 1, ip1jp1 = ij + iall + 1, ijp1 = ij + iall;
          int im1j = ij - 1, ijm1 = ij - iall;
          if (im1j < 1) im1j = 1;
          if (ijm1 < 1) ijm1 = 1;
          double q0 = R3(q, ij, k, l);
          double q_min_AI = fmin2(fmin2(fmin2(q0, R3(q, ijm1, k, l)), R3(q, ip1j, k, l)), R3(q, ip1jp1, k, l));
          double q_max_AI = fmax2(fmax2(fmax2(q0, R3(q, ijm1, k, l)), R3(q, ip1j, k, l)), R3(q, ip1jp1, k, l));
          double q_min_AIJ = fmin2(fmin2(fmin2(q0, R3(q, ip1j, k, l)), R3(q, ip1jp1, k, l)), R3(q, ijp1, k, l));
          double q_max_AIJ = fmax2(fmax2(fmax2(q0, R3(q, ip1j, k, l)), R3(q, ip1jp1, k, l)), R3(q, ijp1, k, l));
          double q_min_AJ = fmin2(fmin2(fmin2(q0, R3(q, ip1jp1, k, l)), R3(q, ijp1, k, l)), R3(q, im1j, k, l));
          double q_max_AJ = fmax2(fmax2(fmax2(q0, R3(q, ip1jp1, k, l)), R3(q, ijp1, k, l)), R3(q, im1j, k, l));
          double c1 = R4(cmask, ij, k, l, 1), c2 = R4(cmask, ij, k, l, 2), c3 = R4(cmask, ij, k, l, 3);
          QIN(ij, k, l, I_min, 1) = c1 * q_min_AI + (1.0 - c1) * BIG;
          QIN(ip1j, k, l, I_min, 4) = c1 * BIG + (1.0 - c1) * q_min_AI;
          QIN(ij, k, l, I_max, 1) = c1 * q_max_AI + (1.0 - c1) * (-BIG);
          QIN(ip1j, k, l, I_max, 4) = c1 * (-BIG) + (1.0 - c1) * q_max_AI;
          QIN(ij, k, l, I_min, 2) = c2 * q_min_AIJ + (1.0 - c2) * BIG;
          QIN(ip1jp1, k, l, I_min, 5) = c2 * BIG + (1.0 - c2) * q_min_AIJ;
          QIN(ij, k, l, I_max, 2) = c2 * q_max_AIJ + (1.0 - c2) * (-BIG);
          QIN(ip1jp1, k, l, I_max, 5) = c2 * (-BIG) + (1.0 - c2) * q_max_AIJ;
          QIN(ij, k, l, I_min, 3) = c3 * q_min_AJ + (1.0 - c3) * BIG;
          QIN(ijp1, k, l, I_min, 6) = c3 * BIG + (1.0 - c3) * q_min_AJ;
          QIN(ij, k, l, I_max, 3) = c3 * q_max_AJ + (1.0 - c3) * (-BIG);
          QIN(ijp1, k, l, I_max, 6) = c3 * (-BIG) + (1.0 - c3) * q_max_AJ;
        }
      /* singular point   :192-214 */
      if (have_sgp[l - 1]) {
        int j = gmin - 1, i = gmin - 1;
        int ij = (j - 1) * iall + i, ijp1 = ij + iall, ip1jp1 = ij + iall + 1, ip2jp1 = ij + iall + 2;
        double q0 = R3(q, ij, k, l);
        double q_min_AIJ = fmin2(fmin2(fmin2(q0, R3(q, ip1jp1, k, l)), R3(q, ip2jp1, k, l)), R3(q, ijp1, k, l));
        double q_max_AIJ = fmax2(fmax2(fmax2(q0, R3(q, ip1jp1, k, l)), R3(q, ip2jp1, k, l)), R3(q, ijp1, k, l));
        double c2 = R4(cmask, ij, k, l, 2);
        QIN(ij, k, l, I_min, 2) = c2 * q_min_AIJ + (1.0 - c2) * BIG;
        QIN(ip1jp1, k, l, I_min, 5) = c2 * BIG + (1.0 - c2) * q_min_AIJ;
        QIN(ij, k, l, I_max, 2) = c2 * q_max_AIJ + (1.0 - c2) * (-BIG);
        QIN(ip1jp1, k, l, I_max, 5) = c2 * (-BIG) + (1.0 - c2) * q_max_AIJ;
      }
      /* (iii) allowable range   :219-282 */
      for (int j = gmin; j <= gmax; ++j)
        for (int i = gmin; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i;
          double q0 = R3(q, ij, k, l);
          double qnext_min = q0, qnext_max = q0;
          for (int f = 1; f <= 6; ++f) qnext_min = fmin2(qnext_min, QIN(ij, k, l, I_min, f));
          for (int f = 1; f <= 6; ++f) qnext_max = fmax2(qnext_max, QIN(ij, k, l, I_max, f));
          double chv[7], cm[7];
          for (int f = 1; f <= 6; ++f) {
            chv[f] = R4(ch, ij, k, l, f);
            cm[f] = fmin2(chv[f], 0.0);
          }
          double Cin_sum = cm[1] + cm[2] + cm[3] + cm[4] + cm[5] + cm[6];
          double Cout_sum = chv[1] - cm[1] + chv[2] - cm[2] + chv[3] - cm[3] + chv[4] - cm[4] + chv[5] - cm[5] + chv[6] - cm[6];
          double CQin_min_sum = cm[1] * QIN(ij, k, l, I_min, 1) + cm[2] * QIN(ij, k, l, I_min, 2) + cm[3] * QIN(ij, k, l, I_min, 3)
                              + cm[4] * QIN(ij, k, l, I_min, 4) + cm[5] * QIN(ij, k, l, I_min, 5) + cm[6] * QIN(ij, k, l, I_min, 6);
          double CQin_max_sum = cm[1] * QIN(ij, k, l, I_max, 1) + cm[2] * QIN(ij, k, l, I_max, 2) + cm[3] * QIN(ij, k, l, I_max, 3)
                              + cm[4] * QIN(ij, k, l, I_max, 4) + cm[5] * QIN(ij, k, l, I_max, 5) + cm[6] * QIN(ij, k, l, I_max, 6);
          double zerosw = 0.5 - fsign(0.5, fabs(Cout_sum) - EPS);
          double dv = R3(dd, ij, k, l);
          R4(Qout, ij, k, l, I_min) = (q0 - CQin_max_sum - qnext_max * (1.0 - Cin_sum - Cout_sum + dv)) / (Cout_sum + zerosw) * (1.0 - zerosw) + q0 * zerosw;
          R4(Qout, ij, k, l, I_max) = (q0 - CQin_min_sum - qnext_min * (1.0 - Cin_sum - Cout_sum + dv)) / (Cout_sum + zerosw) * (1.0 - zerosw) + q0 * zerosw;
        }
      /* halo   :288-301 */
      for (int j = 1; j <= iall; ++j)
        for (int i = 1; i <= iall; ++i)
          if (i < gmin || i > gmax || j < gmin || j > gmax) {
            int ij = (j - 1) * iall + i;
            R4(Qout, ij, k, l, I_min) = R3(q, ij, k, l);
            R4(Qout, ij, k, l, I_max) = R3(q, ij, k, l);
          }
    }
  }
  /* poles   :307-363 */
  if (d->have_pl) {
    const int n = 1, gmin_pl = 2, gmax_pl = 6;
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k) {
        for (int v = gmin_pl; v <= gmax_pl; ++v) {
          int ij = v, ijp1 = v + 1, ijm1 = v - 1;
          if (ijp1 == gmax_pl + 1) ijp1 = gmin_pl;
          if (ijm1 == gmin_pl - 1) ijm1 = gmax_pl;
          double q_min_pl = fmin2(fmin2(fmin2(P3(q_pl, n, k, l), P3(q_pl, ij, k, l)), P3(q_pl, ijm1, k, l)), P3(q_pl, ijp1, k, l));
          double q_max_pl = fmax2(fmax2(fmax2(P3(q_pl, n, k, l), P3(q_pl, ij, k, l)), P3(q_pl, ijm1, k, l)), P3(q_pl, ijp1, k, l));
          double c = P3(cmask_pl, ij, k, l);
          QIN_PL(ij, k, l, I_min, 1) = c * q_min_pl + (1.0 - c) * BIG;
          QIN_PL(ij, k, l, I_min, 2) = c * BIG + (1.0 - c) * q_min_pl;
          QIN_PL(ij, k, l, I_max, 1) = c * q_max_pl + (1.0 - c) * (-BIG);
          QIN_PL(ij, k, l, I_max, 2) = c * (-BIG) + (1.0 - c) * q_max_pl;
        }
        double qnext_min_pl = P3(q_pl, n, k, l), qnext_max_pl = P3(q_pl, n, k, l);
        for (int v = gmin_pl; v <= gmax_pl; ++v) {
          qnext_min_pl = fmin2(qnext_min_pl, QIN_PL(v, k, l, I_min, 1));
          qnext_max_pl = fmax2(qnext_max_pl, QIN_PL(v, k, l, I_max, 1));
        }
        double Cin_sum_pl = 0.0, Cout_sum_pl = 0.0, CQin_max_sum_pl = 0.0, CQin_min_sum_pl = 0.0;
        for (int v = gmin_pl; v <= gmax_pl; ++v) {
          double ch_masked = P3(cmask_pl, v, k, l) * P3(ch_pl, v, k, l);
          Cin_sum_pl = Cin_sum_pl + ch_masked;
          Cout_sum_pl = Cout_sum_pl - ch_masked + P3(ch_pl, v, k, l);
          CQin_min_sum_pl = CQin_min_sum_pl + ch_masked * QIN_PL(v, k, l, I_min, 1);
          CQin_max_sum_pl = CQin_max_sum_pl + ch_masked * QIN_PL(v, k, l, I_max, 1);
        }
        double zerosw = 0.5 - fsign(0.5, fabs(Cout_sum_pl) - EPS);
        double qn = P3(q_pl, n, k, l), dn = P3(d_pl, n, k, l);
        P4(Qout_pl, n, k, l, I_min) = (qn - CQin_max_sum_pl - qnext_max_pl * (1.0 - Cin_sum_pl - Cout_sum_pl + dn)) / (Cout_sum_pl + zerosw) * (1.0 - zerosw) + qn * zerosw;
        P4(Qout_pl, n, k, l, I_max) = (qn - CQin_min_sum_pl - qnext_min_pl * (1.0 - Cin_sum_pl - Cout_sum_pl + dn)) / (Cout_sum_pl + zerosw) * (1.0 - zerosw) + qn * zerosw;
      }
  }
  /* :367-373 */
  for (int mm = 1; mm <= 2; ++mm)
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int v = 2; v <= 6; ++v) P4(Qout_pl, v, k, l, mm) = 0.0;
  memcpy(Qout_prev, Qout, sizeof(double) * (size_t)gall * kall * lall * 2);
  memcpy(Qout_prev_pl, Qout_pl, sizeof(double) * (size_t)gall_pl * kall * lall_pl * 2);
  if (Qout_post) {
    memcpy(Qout, Qout_post, sizeof(double) * (size_t)gall * kall * lall * 2);
    memcpy(Qout_pl, Qout_post_pl, sizeof(double) * (size_t)gall_pl * kall * lall_pl * 2);
  } else {
    /* NICAM original: call COMM_data_transfer( Qout, Qout_pl )   :371 */
    orc_comm_single(topo, Qout, Qout_pl, kall, 2);
  }
  /* apply   :378-410 */
  for (int l = 1; l <= lall; ++l)
    for (int k = 1; k <= kall; ++k)
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i, ip1j = ij + 1, ip1jp1 = ij + iall + 1, ijp1 = ij + iall;
          double c1 = R4(cmask, ij, k, l, 1), c2 = R4(cmask, ij, k, l, 2), c3 = R4(cmask, ij, k, l, 3);
          double v;
          v = R4(q_a, ij, k, l, 1);
          v = c1 * fmin2(fmax2(v, QIN(ij, k, l, I_min, 1)), QIN(ij, k, l, I_max, 1))
            + (1.0 - c1) * fmin2(fmax2(v, QIN(ip1j, k, l, I_min, 4)), QIN(ip1j, k, l, I_max, 4));
          v = c1 * fmax2(fmin2(v, R4(Qout, ip1j, k, l, I_max)), R4(Qout, ip1j, k, l, I_min))
            + (1.0 - c1) * fmax2(fmin2(v, R4(Qout, ij, k, l, I_max)), R4(Qout, ij, k, l, I_min));
          R4(q_a, ij, k, l, 1) = v;
          R4(q_a, ip1j, k, l, 4) = v;
          v = R4(q_a, ij, k, l, 2);
          v = c2 * fmin2(fmax2(v, QIN(ij, k, l, I_min, 2)), QIN(ij, k, l, I_max, 2))
            + (1.0 - c2) * fmin2(fmax2(v, QIN(ip1jp1, k, l, I_min, 5)), QIN(ip1jp1, k, l, I_max, 5));
          v = c2 * fmax2(fmin2(v, R4(Qout, ip1jp1, k, l, I_max)), R4(Qout, ip1jp1, k, l, I_min))
            + (1.0 - c2) * fmax2(fmin2(v, R4(Qout, ij, k, l, I_max)), R4(Qout, ij, k, l, I_min));
          R4(q_a, ij, k, l, 2) = v;
          R4(q_a, ip1jp1, k, l, 5) = v;
          v = R4(q_a, ij, k, l, 3);
          v = c3 * fmin2(fmax2(v, QIN(ij, k, l, I_min, 3)), QIN(ij, k, l, I_max, 3))
            + (1.0 - c3) * fmin2(fmax2(v, QIN(ijp1, k, l, I_min, 6)), QIN(ijp1, k, l, I_max, 6));
          v = c3 * fmax2(fmin2(v, R4(Qout, ijp1, k, l, I_max)), R4(Qout, ijp1, k, l, I_min))
            + (1.0 - c3) * fmax2(fmin2(v, R4(Qout, ij, k, l, I_max)), R4(Qout, ij, k, l, I_min));
          R4(q_a, ij, k, l, 3) = v;
          R4(q_a, ijp1, k, l, 6) = v;
        }
  /* poles apply   :412-425 */
  if (d->have_pl) {
    const int n = 1;
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int v = 2; v <= 6; ++v) {
          double c = P3(cmask_pl, v, k, l);
          double x = P3(q_a_pl, v, k, l);
          x = c * fmin2(fmax2(x, QIN_PL(v, k, l, I_min, 1)), QIN_PL(v, k, l, I_max, 1))
            + (1.0 - c) * fmin2(fmax2(x, QIN_PL(v, k, l, I_min, 2)), QIN_PL(v, k, l, I_max, 2));
          x = c * fmax2(fmin2(x, P4(Qout_pl, v, k, l, I_max)), P4(Qout_pl, v, k, l, I_min))
            + (1.0 - c) * fmax2(fmin2(x, P4(Qout_pl, n, k, l, I_max)), P4(Qout_pl, n, k, l, I_min));
          P3(q_a_pl, v, k, l) = x;
        }
  }
  free(Qin); free(Qin_pl); free(Qout); free(Qout_pl);
}

/* ------------------------------------------------------------------------- */
void orc_vertical_limiter_thuburn(const orc_dims *d,
                                  double *q_h, double *q_h_pl,
                                  const double *q, const double *q_pl,
                                  const double *dd, const double *d_pl,
                                  const double *ck, const double *ck_pl) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int kmin = d->kmin, kmax = d->kmax;
  const double EPS = DBL_EPSILON, BIG = DBL_MAX;
  double *Qout_min_km1 = calloc(gall, sizeof(double));
  double *Qout_max_km1 = calloc(gall, sizeof(double));
  for (int l = 1; l <= lall; ++l) {
    for (int g = 1; g <= gall; ++g) {
      int k = kmin; /* peeling   :107-142 */
      double inflagL = 0.5 - fsign(0.5, R4(ck, g, k, l, 1));
      double inflagU = 0.5 + fsign(0.5, R4(ck, g, k + 1, l, 1));
      double qk = R3(q, g, k, l), qm = R3(q, g, k - 1, l), qp = R3(q, g, k + 1, l);
      double Qin_minL = fmin2(qk, qm) + (1.0 - inflagL) * BIG;
      double Qin_minU = fmin2(qk, qp) + (1.0 - inflagU) * BIG;
      double Qin_maxL = fmax2(qk, qm) - (1.0 - inflagL) * BIG;
      double Qin_maxU = fmax2(qk, qp) - (1.0 - inflagU) * BIG;
      double qnext_min = fmin2(fmin2(Qin_minL, Qin_minU), qk);
      double qnext_max = fmax2(fmax2(Qin_maxL, Qin_maxU), qk);
      double ck1 = R4(ck, g, k, l, 1), ck2 = R4(ck, g, k, l, 2);
      double Cin = inflagL * ck1 + inflagU * ck2;
      double Cout = (1.0 - inflagL) * ck1 + (1.0 - inflagU) * ck2;
      double CQin_min = inflagL * ck1 * Qin_minL + inflagU * ck2 * Qin_minU;
      double CQin_max = inflagL * ck1 * Qin_maxL + inflagU * ck2 * Qin_maxU;
      double zerosw = 0.5 - fsign(0.5, fabs(Cout) - EPS);
      double dv = R3(dd, g, k, l);
      double Qout_min_k = ((qk - qnext_max) + qnext_max * (Cin + Cout - dv) - CQin_max) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
      double Qout_max_k = ((qk - qnext_min) + qnext_min * (Cin + Cout - dv) - CQin_min) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
      Qout_min_km1[g - 1] = Qout_min_k;
      Qout_max_km1[g - 1] = Qout_max_k;
    }
    for (int k = kmin + 1; k <= kmax; ++k) { /* :145-186 */
      for (int g = 1; g <= gall; ++g) {
        double inflagL = 0.5 - fsign(0.5, R4(ck, g, k, l, 1));
        double inflagU = 0.5 + fsign(0.5, R4(ck, g, k + 1, l, 1));
        double qk = R3(q, g, k, l), qm = R3(q, g, k - 1, l), qp = R3(q, g, k + 1, l);
        double Qin_minL = fmin2(qk, qm) + (1.0 - inflagL) * BIG;
        double Qin_minU = fmin2(qk, qp) + (1.0 - inflagU) * BIG;
        double Qin_maxL = fmax2(qk, qm) - (1.0 - inflagL) * BIG;
        double Qin_maxU = fmax2(qk, qp) - (1.0 - inflagU) * BIG;
        double qnext_min = fmin2(fmin2(Qin_minL, Qin_minU), qk);
        double qnext_max = fmax2(fmax2(Qin_maxL, Qin_maxU), qk);
        double ck1 = R4(ck, g, k, l, 1), ck2 = R4(ck, g, k, l, 2);
        double Cin = inflagL * ck1 + inflagU * ck2;
        double Cout = (1.0 - inflagL) * ck1 + (1.0 - inflagU) * ck2;
        double CQin_min = inflagL * ck1 * Qin_minL + inflagU * ck2 * Qin_minU;
        double CQin_max = inflagL * ck1 * Qin_maxL + inflagU * ck2 * Qin_maxU;
        double zerosw = 0.5 - fsign(0.5, fabs(Cout) - EPS);
        double dv = R3(dd, g, k, l);
        double Qout_min_k = ((qk - qnext_max) + qnext_max * (Cin + Cout - dv) - CQin_max) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
        double Qout_max_k = ((qk - qnext_min) + qnext_min * (Cin + Cout - dv) - CQin_min) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
        double qh = R3(q_h, g, k, l);
        R3(q_h, g, k, l) = inflagL * fmax2(fmin2(qh, Qout_max_km1[g - 1]), Qout_min_km1[g - 1])
                         + (1.0 - inflagL) * fmax2(fmin2(qh, Qout_max_k), Qout_min_k);
        Qout_min_km1[g - 1] = Qout_min_k;
        Qout_max_km1[g - 1] = Qout_max_k;
      }
    }
  }
  if (d->have_pl) { /* :191-238 */
    double *Qout_min_pl = calloc((size_t)gall_pl * kall, sizeof(double));
    double *Qout_max_pl = calloc((size_t)gall_pl * kall, sizeof(double));
#define QP(a, g, k) a[((size_t)(k)-1) * gall_pl + ((g)-1)]
    for (int l = 1; l <= lall_pl; ++l) {
      for (int k = kmin; k <= kmax; ++k)
        for (int g = 1; g <= gall_pl; ++g) {
          double inflagL = 0.5 - fsign(0.5, P4(ck_pl, g, k, l, 1));
          double inflagU = 0.5 + fsign(0.5, P4(ck_pl, g, k + 1, l, 1));
          double qk = P3(q_pl, g, k, l), qm = P3(q_pl, g, k - 1, l), qp = P3(q_pl, g, k + 1, l);
          double Qin_minL = fmin2(qk, qm) + (1.0 - inflagL) * BIG;
          double Qin_minU = fmin2(qk, qp) + (1.0 - inflagU) * BIG;
          double Qin_maxL = fmax2(qk, qm) - (1.0 - inflagL) * BIG;
          double Qin_maxU = fmax2(qk, qp) - (1.0 - inflagU) * BIG;
          double qnext_min = fmin2(fmin2(Qin_minL, Qin_minU), qk);
          double qnext_max = fmax2(fmax2(Qin_maxL, Qin_maxU), qk);
          double ck1 = P4(ck_pl, g, k, l, 1), ck2 = P4(ck_pl, g, k, l, 2);
          double Cin = inflagL * (ck1) + inflagU * (ck2);
          double Cout = (1.0 - inflagL) * (ck1) + (1.0 - inflagU) * (ck2);
          double CQin_max = inflagL * (ck1 * Qin_maxL) + inflagU * (ck2 * Qin_maxU);
          double CQin_min = inflagL * (ck1 * Qin_minL) + inflagU * (ck2 * Qin_minU);
          double zerosw = 0.5 - fsign(0.5, fabs(Cout) - EPS);
          double dv = P3(d_pl, g, k, l);
          QP(Qout_min_pl, g, k) = ((qk - qnext_max) + qnext_max * (Cin + Cout - dv) - CQin_max) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
          QP(Qout_max_pl, g, k) = ((qk - qnext_min) + qnext_min * (Cin + Cout - dv) - CQin_min) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
        }
      for (int k = kmin + 1; k <= kmax; ++k)
        for (int g = 1; g <= gall_pl; ++g) {
          double inflagL = 0.5 - fsign(0.5, P4(ck_pl, g, k, l, 1));
          double qh = P3(q_h_pl, g, k, l);
          P3(q_h_pl, g, k, l) = inflagL * fmax2(fmin2(qh, QP(Qout_max_pl, g, k - 1)), QP(Qout_min_pl, g, k - 1))
                              + (1.0 - inflagL) * fmax2(fmin2(qh, QP(Qout_max_pl, g, k)), QP(Qout_min_pl, g, k));
        }
    }
#undef QP
    free(Qout_min_pl); free(Qout_max_pl);
  }
  free(Qout_min_km1); free(Qout_max_km1);
}
