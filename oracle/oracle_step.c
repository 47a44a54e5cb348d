/*
 * CPU oracle: the composed tracer step.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference ships the three kernels and the halo exchange but never
 * composes them, and has no gradient apply, remap, Courant number / mask or
 * rhogq update (parity unpinned).  The composition below follows NICAM's
 * tracer scheme as described in docs/NICAM/src/20_intro_nicam.tex:368-429
 * (Miura 2007 upwind remap) and the argument meanings in
 * docs/NICAM/src/36_horiz_adv_limiter.tex:121-127 and 34_vert_adv_limiter.tex:
 *
 *   horizontal sub-step (full dt)
 *     flx_h, GRD_xc   = horizontal_flux(rhog, rhogv)
 *     ch              = flx_h / rhog                 (per face, 6 per cell)
 *     cmask           = 0.5 - sign(0.5, ch - EPS)    (1 where the face flow enters the cell)
 *     q               = rhogq / rhog
 *     grad q          = sum_n coef_grad(n) q(nb_n)   (OPRT_gradient_setup stencil,
 *                                                     dyn_metrics/src/mod_oprt.f90:499-734)
 *     halo fill of grad q (COMM_data_transfer)
 *     q_a(face)       = q(up) + grad q(up) . (GRD_xc(face) - GRD_x(up)),  up = upwind cell
 *     q_a             = horizontal_limiter_thuburn(q_a, q, d=0, ch, cmask)  (Qout halo by COMM)
 *     rhogq          -= sum_m flx_h(m) q_a(m) ;  rhog -= sum_m flx_h(m)
 *   vertical sub-step (full dt, after the horizontal one)
 *     q               = rhogq / rhog ; ghost levels copy kmin / kmax
 *     ck(k,1)         = -rhogw(k)   dt rdgz(k) / rhog(k)
 *     ck(k,2)         =  rhogw(k+1) dt rdgz(k) / rhog(k)
 *     q_h(k)          = afact(k) q(k) + bfact(k) q(k-1)   (value at face k-1/2)
 *     q_h             = vertical_limiter_thuburn(q_h, q, d=0, ck)
 *     rhogq(k)       -= (rhogw(k+1) q_h(k+1) - rhogw(k) q_h(k)) dt rdgz(k)
 *     rhog(k)        -= (rhogw(k+1) - rhogw(k)) dt rdgz(k)
 *   halo fill of rhog and rhogq (COMM_data_transfer)
 *
 * With d = 0 the Thuburn consistency 1 - Cin - Cout + d = rhog_new/rhog_old
 * holds by construction, so a constant mixing ratio stays constant.
 */
#include "icoadv_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void orc_comm_single(const orc_topo *t, double *var, double *var_pl, int kmax, int vmax);

#define R3(a, ij, k, l) a[((size_t)((l)-1) * kall + ((k)-1)) * gall + ((ij)-1)]
#define R4(a, ij, k, l, m) a[(((size_t)((m)-1) * lall + ((l)-1)) * kall + ((k)-1)) * gall + ((ij)-1)]
#define R5(a, ij, k, l, m, n) \
  a[((((size_t)((n)-1) * 3 + ((m)-1)) * lall + ((l)-1)) * kall + ((k)-1)) * gall + ((ij)-1)]
#define P3(a, v, k, l) a[((size_t)((l)-1) * kall + ((k)-1)) * gall_pl + ((v)-1)]
#define P4(a, v, k, l, m) a[(((size_t)((m)-1) * lall_pl + ((l)-1)) * kall + ((k)-1)) * gall_pl + ((v)-1)]
/* GRD_x(gall,1,lall,3) */
#define GX(ij, l, x) GRD_x[(((size_t)((x)-1) * lall + ((l)-1))) * gall + ((ij)-1)]
#define GX_PL(v, l, x) GRD_x_pl[(((size_t)((x)-1) * lall_pl + ((l)-1))) * gall_pl + ((v)-1)]
/* coef_grad(gall,0:6,3,lall), coef_grad_pl(0:5,3,lall_pl) */
#define CG(ij, n, x, l) coef_grad[((((size_t)((l)-1) * 3 + ((x)-1)) * 7 + (n))) * gall + ((ij)-1)]
#define CG_PL(n, x, l) coef_grad_pl[(((size_t)((l)-1) * 3 + ((x)-1)) * 6 + (n))]

static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

void orc_gradient(const orc_dims *d, const int *have_sgp, double *grad, double *grad_pl,
                  const double *q, const double *q_pl,
                  const double *coef_grad, const double *coef_grad_pl) {
  (void)have_sgp;
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int gmin = d->gmin, gmax = d->gmax, iall = d->gall_1d;
  memset(grad, 0, sizeof(double) * (size_t)gall * kall * lall * 3);
  for (int l = 1; l <= lall; ++l)
    for (int k = 1; k <= kall; ++k)
      for (int j = gmin; j <= gmax; ++j)
        for (int i = gmin; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i;
          int nb[7] = {ij, ij + 1, ij + iall + 1, ij + iall, ij - 1, ij - iall - 1, ij - iall};
          for (int x = 1; x <= 3; ++x) {
            double s = CG(ij, 0, x, l) * R3(q, nb[0], k, l);
            for (int n = 1; n <= 6; ++n) s = s + CG(ij, n, x, l) * R3(q, nb[n], k, l);
            R4(grad, ij, k, l, x) = s;
          }
        }
  if (d->have_pl) {
    memset(grad_pl, 0, sizeof(double) * (size_t)gall_pl * kall * lall_pl * 3);
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int x = 1; x <= 3; ++x) {
          double s = CG_PL(0, x, l) * P3(q_pl, 1, k, l);
          for (int v = 2; v <= 6; ++v) s = s + CG_PL(v - 1, x, l) * P3(q_pl, v, k, l);
          P4(grad_pl, 1, k, l, x) = s;
        }
  }
}

void orc_courant(const orc_dims *d, double *ch, double *ch_pl, double *cmask, double *cmask_pl,
                 const double *flx_h, const double *flx_h_pl, const double *rho, const double *rho_pl) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const double EPS = DBL_EPSILON;
  for (int m = 1; m <= 6; ++m)
    for (int l = 1; l <= lall; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int ij = 1; ij <= gall; ++ij) {
          double c = R4(flx_h, ij, k, l, m) / R3(rho, ij, k, l);
          R4(ch, ij, k, l, m) = c;
          R4(cmask, ij, k, l, m) = 0.5 - fsign(0.5, c - EPS);
        }
  if (d->have_pl)
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int v = 1; v <= gall_pl; ++v) {
          double c = (v == 1) ? 0.0 : P3(flx_h_pl, v, k, l) / P3(rho_pl, 1, k, l);
          P3(ch_pl, v, k, l) = c;
          P3(cmask_pl, v, k, l) = 0.5 - fsign(0.5, c - EPS);
        }
}

void orc_remap(const orc_dims *d, double *q_a, double *q_a_pl,
               const double *q, const double *q_pl, const double *grad, const double *grad_pl,
               const double *cmask, const double *cmask_pl,
               const double *GRD_xc, const double *GRD_xc_pl,
               const double *GRD_x, const double *GRD_x_pl) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int gmin = d->gmin, gmax = d->gmax, iall = d->gall_1d;
  memset(q_a, 0, sizeof(double) * (size_t)gall * kall * lall * 6);
  for (int l = 1; l <= lall; ++l)
    for (int k = 1; k <= kall; ++k)
      for (int j = gmin - 1; j <= gmax; ++j)
        for (int i = gmin - 1; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i;
          int nbs[4] = {0, ij + 1, ij + iall + 1, ij + iall};
          for (int m = 1; m <= 3; ++m) {
            int nb = nbs[m];
            double c = R4(cmask, ij, k, l, m);
            double vu = R3(q, nb, k, l)
                      + R4(grad, nb, k, l, 1) * (R5(GRD_xc, ij, k, l, m, 1) - GX(nb, l, 1))
                      + R4(grad, nb, k, l, 2) * (R5(GRD_xc, ij, k, l, m, 2) - GX(nb, l, 2))
                      + R4(grad, nb, k, l, 3) * (R5(GRD_xc, ij, k, l, m, 3) - GX(nb, l, 3));
            double vs = R3(q, ij, k, l)
                      + R4(grad, ij, k, l, 1) * (R5(GRD_xc, ij, k, l, m, 1) - GX(ij, l, 1))
                      + R4(grad, ij, k, l, 2) * (R5(GRD_xc, ij, k, l, m, 2) - GX(ij, l, 2))
                      + R4(grad, ij, k, l, 3) * (R5(GRD_xc, ij, k, l, m, 3) - GX(ij, l, 3));
            double v = c * vu + (1.0 - c) * vs;
            R4(q_a, ij, k, l, m) = v;
            R4(q_a, nb, k, l, m + 3) = v;
          }
        }
  if (d->have_pl) {
    memset(q_a_pl, 0, sizeof(double) * (size_t)gall_pl * kall * lall_pl);
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int v = 2; v <= 6; ++v) {
          double c = P3(cmask_pl, v, k, l);
          double vu = P3(q_pl, v, k, l)
                    + P4(grad_pl, v, k, l, 1) * (P4(GRD_xc_pl, v, k, l, 1) - GX_PL(v, l, 1))
                    + P4(grad_pl, v, k, l, 2) * (P4(GRD_xc_pl, v, k, l, 2) - GX_PL(v, l, 2))
                    + P4(grad_pl, v, k, l, 3) * (P4(GRD_xc_pl, v, k, l, 3) - GX_PL(v, l, 3));
          double vs = P3(q_pl, 1, k, l)
                    + P4(grad_pl, 1, k, l, 1) * (P4(GRD_xc_pl, v, k, l, 1) - GX_PL(1, l, 1))
                    + P4(grad_pl, 1, k, l, 2) * (P4(GRD_xc_pl, v, k, l, 2) - GX_PL(1, l, 2))
                    + P4(grad_pl, 1, k, l, 3) * (P4(GRD_xc_pl, v, k, l, 3) - GX_PL(1, l, 3));
          P3(q_a_pl, v, k, l) = c * vu + (1.0 - c) * vs;
        }
  }
}

/* vertical sub-step for one column of length kall: in/out rhog, rhogq (ntr, stride) */
static void vertical_column(int kall, int kmin, int kmax, double dt,
                            double *rhog, size_t rs, double *rhogq, size_t qs_k, size_t qs_t, int ntr,
                            const double *rhogw, size_t ws, const double *rdgz,
                            const double *afact, const double *bfact, const orc_dims *d1) {
  double *ck = malloc(sizeof(double) * 2 * kall);
  double *q = malloc(sizeof(double) * kall);
  double *qh = malloc(sizeof(double) * kall);
  double *zero = calloc(kall, sizeof(double));
  for (int k = 1; k <= kall; ++k) {
    ck[k - 1] = 0.0;
    ck[kall + k - 1] = 0.0;
  }
  for (int k = kmin; k <= kmax; ++k) {
    double r = rhog[(k - 1) * rs];
    ck[k - 1] = -rhogw[(k - 1) * ws] * dt * rdgz[k - 1] / r;
    ck[kall + k - 1] = rhogw[k * ws] * dt * rdgz[k - 1] / r;
  }
  ck[kall - 1] = -rhogw[(kall - 1) * ws] * dt * rdgz[kall - 1] / rhog[(kall - 1) * rs];
  for (int t = 0; t < ntr; ++t) {
    double *Q = rhogq + t * qs_t;
    for (int k = kmin; k <= kmax; ++k) q[k - 1] = Q[(k - 1) * qs_k] / rhog[(k - 1) * rs];
    q[0] = q[kmin - 1];
    q[kall - 1] = q[kmax - 1];
    for (int k = kmin; k <= kmax + 1 && k <= kall; ++k)
      qh[k - 1] = afact[k - 1] * q[k - 1] + bfact[k - 1] * q[k - 2];
    qh[0] = 0.0;
    orc_vertical_limiter_thuburn(d1, qh, NULL, q, NULL, zero, NULL, ck, NULL);
    for (int k = kmin; k <= kmax; ++k) {
      double fu = rhogw[k * ws] * qh[k], fl = rhogw[(k - 1) * ws] * qh[k - 1];
      Q[(k - 1) * qs_k] = Q[(k - 1) * qs_k] - (fu - fl) * dt * rdgz[k - 1];
    }
    Q[0] = Q[(kmin - 1) * qs_k];
    Q[(kall - 1) * qs_k] = Q[(kmax - 1) * qs_k];
  }
  for (int k = kmin; k <= kmax; ++k)
    rhog[(k - 1) * rs] = rhog[(k - 1) * rs] - (rhogw[k * ws] - rhogw[(k - 1) * ws]) * dt * rdgz[k - 1];
  rhog[0] = rhog[(kmin - 1) * rs];
  rhog[(kall - 1) * rs] = rhog[(kmax - 1) * rs];
  free(ck); free(q); free(qh); free(zero);
}

/* Scratch kept across calls (process lifetime), so that a step does not map and fault its
   temporaries again (at glevel 8 they are gigabytes, which made the CPU time mostly page
   faults).  Slot s holds one buffer that only grows; its contents are not kept meaningful
   between uses.  orc_step is not reentrant. */
enum { SCR_FLX, SCR_XC, SCR_CH, SCR_CM, SCR_ZERO, SCR_TRACER0, SCR_NSLOT = SCR_TRACER0 + 4 * 256 };
static double *scr_ptr[SCR_NSLOT];
static size_t scr_len[SCR_NSLOT];
static double *scratch(int slot, size_t n, int zero) {
  if (scr_len[slot] < n) {
    free(scr_ptr[slot]);
    scr_ptr[slot] = malloc(sizeof(double) * n);
    scr_len[slot] = scr_ptr[slot] ? n : 0;
  }
  if (zero && scr_ptr[slot]) memset(scr_ptr[slot], 0, sizeof(double) * n);
  return scr_ptr[slot];
}

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
              int nthreads) {
  const int gall = d->gall, kall = d->kall, lall = d->lall;
  const int gall_pl = d->gall_pl, lall_pl = d->lall_pl;
  const int gmin = d->gmin, gmax = d->gmax, iall = d->gall_1d;
  const size_t n3 = (size_t)gall * kall * lall, n3p = (size_t)gall_pl * kall * lall_pl;
  int nthr = nthreads > 0 ? nthreads : 1;
  if (nthr > 256) nthr = 256;
  double *flx = scratch(SCR_FLX, n3 * 6, 0), *flx_pl = calloc(n3p, sizeof(double));
  double *xc = scratch(SCR_XC, n3 * 9, 0), *xc_pl = calloc(n3p * 3, sizeof(double));
  double *ch = scratch(SCR_CH, n3 * 6, 0), *ch_pl = calloc(n3p, sizeof(double));
  double *cm = scratch(SCR_CM, n3 * 6, 0), *cm_pl = calloc(n3p, sizeof(double));
  /* the density correction d of the limiter: zero (read only) */
  double *zero = scratch(SCR_ZERO, n3, 1), *zero_pl = calloc(n3p, sizeof(double));
  /* every thread's tracer temporaries, set up before the parallel region */
  for (int th = 0; th < nthr; ++th) {
    scratch(SCR_TRACER0 + 4 * th + 0, n3, 0);
    scratch(SCR_TRACER0 + 4 * th + 1, n3 * 3, 0);
    scratch(SCR_TRACER0 + 4 * th + 2, n3 * 6, 0);
    scratch(SCR_TRACER0 + 4 * th + 3, n3 * 2, 0);
  }
  orc_horizontal_flux(d, have_sgp, flx, flx_pl, xc, xc_pl, rhog, rhog_pl, rhogvx, rhogvx_pl,
                      rhogvy, rhogvy_pl, rhogvz, rhogvz_pl, dt, GRD_xr, GRD_xr_pl,
                      GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl);
  orc_courant(d, ch, ch_pl, cm, cm_pl, flx, flx_pl, rhog, rhog_pl);

#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr)
#endif
  for (int t = 0; t < ntr; ++t) {
#ifdef _OPENMP
    const int th = omp_get_thread_num();
#else
    const int th = 0;
#endif
    double *Q = rhogq + (size_t)t * n3, *Qp = rhogq_pl + (size_t)t * n3p;
    /* the thread's region temporaries (every value the tracer reads is written first, as
       with fresh malloc'd memory); the pole arrays start at zero */
    double *q = scr_ptr[SCR_TRACER0 + 4 * th + 0], *q_pl = calloc(n3p, sizeof(double));
    double *gr = scr_ptr[SCR_TRACER0 + 4 * th + 1], *gr_pl = calloc(n3p * 3, sizeof(double));
    double *qa = scr_ptr[SCR_TRACER0 + 4 * th + 2], *qa_pl = calloc(n3p, sizeof(double));
    double *qo = scr_ptr[SCR_TRACER0 + 4 * th + 3], *qo_pl = calloc(n3p * 2, sizeof(double));
    for (size_t i = 0; i < n3; ++i) q[i] = Q[i] / rhog[i];
    if (d->have_pl)
      for (size_t i = 0; i < n3p; ++i) q_pl[i] = Qp[i] / rhog_pl[i];
    orc_gradient(d, have_sgp, gr, gr_pl, q, q_pl, coef_grad, coef_grad_pl);
    orc_comm_single(topo, gr, gr_pl, kall, 3);
    orc_remap(d, qa, qa_pl, q, q_pl, gr, gr_pl, cm, cm_pl, xc, xc_pl, GRD_x, GRD_x_pl);
    orc_horizontal_limiter_thuburn(d, have_sgp, qa, qa_pl, q, q_pl, zero, zero_pl, ch, ch_pl,
                                   cm, cm_pl, qo, qo_pl, NULL, NULL, topo);
    for (int l = 1; l <= lall; ++l)
      for (int k = 1; k <= kall; ++k)
        for (int j = gmin; j <= gmax; ++j)
          for (int i = gmin; i <= gmax; ++i) {
            int ij = (j - 1) * iall + i;
            double s = R4(flx, ij, k, l, 1) * R4(qa, ij, k, l, 1);
            for (int m = 2; m <= 6; ++m) s = s + R4(flx, ij, k, l, m) * R4(qa, ij, k, l, m);
            R3(Q, ij, k, l) = R3(Q, ij, k, l) - s;
          }
    if (d->have_pl)
      for (int l = 1; l <= lall_pl; ++l)
        for (int k = 1; k <= kall; ++k) {
          double s = P3(flx_pl, 2, k, l) * P3(qa_pl, 2, k, l);
          for (int v = 3; v <= 6; ++v) s = s + P3(flx_pl, v, k, l) * P3(qa_pl, v, k, l);
          P3(Qp, 1, k, l) = P3(Qp, 1, k, l) - s;
        }
    free(q_pl); free(gr_pl); free(qa_pl); free(qo_pl);
  }
  free(zero_pl);
  /* density after the horizontal sub-step (columns are independent: threads over regions
     and levels, each value computed by the same operations as in a serial loop) */
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
#endif
  for (int l = 1; l <= lall; ++l)
    for (int k = 1; k <= kall; ++k)
      for (int j = gmin; j <= gmax; ++j)
        for (int i = gmin; i <= gmax; ++i) {
          int ij = (j - 1) * iall + i;
          double s = R4(flx, ij, k, l, 1);
          for (int m = 2; m <= 6; ++m) s = s + R4(flx, ij, k, l, m);
          R3(rhog, ij, k, l) = R3(rhog, ij, k, l) - s;
        }
  if (d->have_pl)
    for (int l = 1; l <= lall_pl; ++l)
      for (int k = 1; k <= kall; ++k) {
        double s = P3(flx_pl, 2, k, l);
        for (int v = 3; v <= 6; ++v) s = s + P3(flx_pl, v, k, l);
        P3(rhog_pl, 1, k, l) = P3(rhog_pl, 1, k, l) - s;
      }
  /* vertical sub-step, interior columns and pole centres */
  orc_dims d1 = {0};
  d1.kall = kall; d1.kmin = d->kmin; d1.kmax = d->kmax;
  d1.gall = 1; d1.lall = 1; d1.have_pl = 0; d1.gall_pl = 6; d1.lall_pl = 2;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
#endif
  for (int l = 1; l <= lall; ++l)
    for (int j = gmin; j <= gmax; ++j)
      for (int i = gmin; i <= gmax; ++i) {
        int ij = (j - 1) * iall + i;
        size_t base = ((size_t)(l - 1) * kall) * gall + (ij - 1);
        vertical_column(kall, d->kmin, d->kmax, dt, rhog + base, gall, rhogq + base, gall, n3, ntr,
                        rhogw + base, gall, rdgz, afact, bfact, &d1);
      }
  if (d->have_pl)
    for (int l = 1; l <= lall_pl; ++l) {
      size_t base = ((size_t)(l - 1) * kall) * gall_pl;
      vertical_column(kall, d->kmin, d->kmax, dt, rhog_pl + base, gall_pl, rhogq_pl + base, gall_pl, n3p, ntr,
                      rhogw_pl + base, gall_pl, rdgz, afact, bfact, &d1);
    }
  /* halo fill of the state */
  orc_comm_single(topo, rhog, rhog_pl, kall, 1);
  orc_comm_single(topo, rhogq, rhogq_pl, kall, ntr);
  free(flx_pl); free(xc_pl); free(ch_pl); free(cm_pl);
}
