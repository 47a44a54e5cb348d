// Composed-step launch interface (plain FP64 path).
#pragma once

#include "plain_kernels.cuh"

namespace icoadv {

struct DevPlan {
  int n;
  const int *dst, *src;
};

// Device pointers used by one composed step: metrics, step geometry, scratch.
struct StepCtx {
  Dims D;
  Geo<double> geo;
  DevPlan plan;
  const double *GRD_x, *GRD_x_pl, *cg, *cg_pl, *rdgz, *afact, *bfact;
  // shared per step
  double *flx, *flx_pl, *xc, *xc_pl, *ch, *ch_pl, *cm, *cm_pl, *zero, *zero_pl;
  // per tracer
  double *q, *q_pl, *grad, *grad_pl, *qa, *qa_pl, *qout, *qout_pl, *qin_pl;
};

// Pieces of the plain step, also used by the adjoint's forward recompute.
void launch_courant(const StepCtx &S, const double *rhog, const double *rhog_pl, cudaStream_t st);  // flx -> ch, cm
void launch_divide(const StepCtx &S, const double *Q, const double *Qp, const double *rhog, const double *rhog_pl,
                   cudaStream_t st);                                  // q = Q / rhog
void launch_gradient(const StepCtx &S, cudaStream_t st);             // q -> grad, halo filled
void launch_remap(const StepCtx &S, cudaStream_t st);                // q, grad -> qa
void launch_update_h(const StepCtx &S, const double *qa, const double *qa_pl, double *Q, double *Qp,
                     cudaStream_t st);                                // Q -= sum flx qa (interior, pole centres)
void launch_update_rho(const StepCtx &S, double *rho, double *rho_pl, cudaStream_t st);  // rho -= sum flx

int step_plain(StepCtx &S, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
               const double *vx, const double *vx_pl, const double *vy, const double *vy_pl, const double *vz,
               const double *vz_pl, const double *w, const double *w_pl, cudaStream_t st, long long &launches);

}  // namespace icoadv
