// Adjoint (reverse mode) of the plain FP64 step.
#pragma once

#include "step.cuh"

namespace icoadv {

// Device scratch of one adjoint step, besides the forward scratch of StepCtx.
struct AdjScratch {
  double *rh, *rh_pl;          // rhog after the horizontal sub-step
  double *qa1, *qa1_pl;        // limited face values of the current tracer
  double *Qh, *Qh_pl;          // rhogq after the horizontal sub-step, current tracer
  double *a_q, *a_q_pl;        // adjoint of q = rhogq / rhog, current tracer
  double *aT;                  // triangle adjoints of horizontal_flux (8 fields; aliases qa1 | Qh | a_q)
  double *a_flx, *a_flx_pl, *a_xc, *a_xc_pl, *a_ch, *a_ch_pl, *a_rh, *a_rh_pl;
  double *a_gr, *a_gr_pl, *a_qo, *a_qo_pl;
};

// One adjoint step.  In: the step's input state (rhog, rhogq and their pole
// arrays, unchanged) and the fields; a_rhog / a_rhogq hold the adjoint of the
// step's output on entry and the adjoint of its input on return; the wind
// adjoints a_vx / a_vy / a_vz (+ pole arrays) are accumulated.
int step_adjoint(StepCtx &S, const AdjScratch &A, int ntr, double dt, const double *rhog, const double *rhog_pl,
                 const double *rhogq, const double *rhogq_pl, const double *vx, const double *vx_pl,
                 const double *vy, const double *vy_pl, const double *vz, const double *vz_pl, const double *w,
                 const double *w_pl, double *a_rhog, double *a_rhog_pl, double *a_rhogq, double *a_rhogq_pl,
                 double *a_vx, double *a_vx_pl, double *a_vy, double *a_vy_pl, double *a_vz, double *a_vz_pl,
                 cudaStream_t st, long long &launches);

}  // namespace icoadv
