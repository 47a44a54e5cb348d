// The composed tracer step, plain FP64 path: the reference kernels chained with
// the pieces the reference leaves out (Courant numbers, gradient, remap,
// rhogq update, vertical flux), one kernel each, tracer by tracer.  This is
// the "plain per-tracer" GPU path; the batched path is fast_kernels.cu.
//
// The composition (horizontal sub-step, then vertical sub-step, then the halo
// fill of the state) and every formula match the CPU oracle's definition of
// the step; compiled with --fmad=false the FP64 results equal it bit for bit.
//
//   ch    = flx_h / rhog,  cmask = 0.5 - sign(0.5, ch - EPS)
//   q     = rhogq / rhog
//   grad  = sum_n coef_grad(n) q(nb_n)   (stencil of dyn_metrics/src/mod_oprt.f90:499-734)
//   q_a   = q(up) + grad(up).(GRD_xc - GRD_x(up)), blended by cmask (Miura 2007 remap,
//           docs/NICAM/src/20_intro_nicam.tex:368-429)
//   q_a   = horizontal_limiter_thuburn(q_a, q, 0, ch, cmask) with the Qout halo fill
//   rhogq -= sum_m flx_h(m) q_a(m);  rhog -= sum_m flx_h(m)
//   vertical: ck from rhogw, q_h by linear interpolation, vertical_limiter_thuburn,
//           rhogq -= d/dz(rhogw q_h) dt, rhog -= d/dz(rhogw) dt
#include <cuda_runtime.h>

#include <cfloat>

#include "step.cuh"

namespace icoadv {

__device__ __forceinline__ double sgn(double a, double b) { return copysign(fabs(a), b); }

// ch, cmask for every (face, cell, level, region); poles: ring faces v = 2..6, ch(1) = 0
__global__ void k_courant(int n3, const double *flx, const double *rho, double *ch, double *cm) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6LL * n3) return;
  const double c = flx[t] / rho[t % n3];
  ch[t] = c;
  cm[t] = 0.5 - sgn(0.5, c - DBL_EPSILON);
}
__global__ void k_courant_pl(int kall, const double *flx_pl, const double *rho_pl, double *ch_pl, double *cm_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall * kGallPl) return;
  const int v = t % kGallPl, kl = t / kGallPl;
  const double c = (v == 0) ? 0.0 : flx_pl[t] / rho_pl[kl * kGallPl];
  ch_pl[t] = c;
  cm_pl[t] = 0.5 - sgn(0.5, c - DBL_EPSILON);
}

// q = rhogq / rhog (regions and poles in one launch)
__global__ void k_divide(long long n3, int n3p, const double *Q, const double *rho, const double *Qp,
                         const double *rhop, double *q, double *qp) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n3) q[t] = Q[t] / rho[t];
  else if (t < n3 + n3p) qp[t - n3] = Qp[t - n3] / rhop[t - n3];
}

// gradient at interior cells, 0 elsewhere; coef_grad(gall,0:6,3,lall)
__global__ void k_gradient(Dims D, const double *q, const double *cg, double *grad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  if (i < D.gmin || i > D.gmax || j < D.gmin || j > D.gmax) {
    for (int x = 0; x < 3; ++x) grad[x * fs + off + c] = 0.0;
    return;
  }
  const int nb[7] = {c, c + 1, c + G + 1, c + G, c - 1, c - G - 1, c - G};
  const double *qs = q + off;
  for (int x = 0; x < 3; ++x) {
    const double *cx = cg + ((size_t)l * 3 + x) * 7 * D.gall + c;
    double s = cx[0] * qs[nb[0]];
    for (int n = 1; n <= 6; ++n) s = s + cx[(size_t)n * D.gall] * qs[nb[n]];
    grad[x * fs + off + c] = s;
  }
}
__global__ void k_gradient_pl(int kall, const double *q_pl, const double *cg_pl, double *grad_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const int l = t / kall;
  const size_t off = (size_t)t * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  for (int x = 0; x < 3; ++x) {
    const double *cx = cg_pl + ((size_t)l * 3 + x) * 6;
    double s = cx[0] * q_pl[off];
    for (int v = 2; v <= 6; ++v) s = s + cx[v - 1] * q_pl[off + v - 1];
    for (int v = 0; v < kGallPl; ++v) grad_pl[x * fsp + off + v] = (v == 0) ? s : 0.0;
  }
}

// upwind remap of the three faces attached to (i,j) in [gmin-1,gmax]^2
__global__ void k_remap(Dims D, const double *q, const double *grad, const double *cm, const double *xc,
                        const double *GRD_x, double *qa) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  if (i < D.gmin - 1 || i > D.gmax || j < D.gmin - 1 || j > D.gmax) return;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  const size_t gw = (size_t)D.lall * D.gall;
  const int nbs[4] = {0, c + 1, c + G + 1, c + G};
  for (int m = 1; m <= 3; ++m) {
    const int nb = nbs[m];
    const double cc = cm[(size_t)(m - 1) * fs + off + c];
    double vu = q[off + nb], vs = q[off + c];
    for (int x = 0; x < 3; ++x) {
      const double xcv = xc[((size_t)x * 3 + (m - 1)) * fs + off + c];
      vu = vu + grad[x * fs + off + nb] * (xcv - GRD_x[x * gw + (size_t)l * D.gall + nb]);
    }
    for (int x = 0; x < 3; ++x) {
      const double xcv = xc[((size_t)x * 3 + (m - 1)) * fs + off + c];
      vs = vs + grad[x * fs + off + c] * (xcv - GRD_x[x * gw + (size_t)l * D.gall + c]);
    }
    const double v = cc * vu + (1.0 - cc) * vs;
    qa[(size_t)(m - 1) * fs + off + c] = v;
    qa[(size_t)(m + 2) * fs + off + nb] = v;
  }
}
__global__ void k_remap_pl(int kall, const double *q_pl, const double *grad_pl, const double *cm_pl,
                           const double *xc_pl, const double *GRD_x_pl, double *qa_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall * kGallPl) return;
  const int v = t % kGallPl, kl = t / kGallPl, l = kl / kall;
  const size_t off = (size_t)kl * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  if (v == 0) {
    qa_pl[off] = 0.0;
    return;
  }
  const double cc = cm_pl[off + v];
  double vu = q_pl[off + v], vs = q_pl[off];
  for (int x = 0; x < 3; ++x)
    vu = vu + grad_pl[x * fsp + off + v] * (xc_pl[x * fsp + off + v] - GRD_x_pl[((size_t)x * kLallPl + l) * kGallPl + v]);
  for (int x = 0; x < 3; ++x)
    vs = vs + grad_pl[x * fsp + off] * (xc_pl[x * fsp + off + v] - GRD_x_pl[((size_t)x * kLallPl + l) * kGallPl]);
  qa_pl[off + v] = cc * vu + (1.0 - cc) * vs;
}

// rhogq -= sum_m flx_h(m) q_a(m) at interior cells (all levels); pole centres
__global__ void k_update_h(Dims D, const double *flx, const double *qa, double *Q) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  if (i < D.gmin || i > D.gmax || j < D.gmin || j > D.gmax) return;
  const size_t off = (size_t)kl * D.gall + c, fs = (size_t)D.lall * D.kall * D.gall;
  double s = flx[off] * qa[off];
  for (int m = 1; m < 6; ++m) s = s + flx[m * fs + off] * qa[m * fs + off];
  Q[off] = Q[off] - s;
}
__global__ void k_update_h_pl(int kall, const double *flx_pl, const double *qa_pl, double *Qp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const size_t off = (size_t)t * kGallPl;
  double s = flx_pl[off + 1] * qa_pl[off + 1];
  for (int v = 3; v <= 6; ++v) s = s + flx_pl[off + v - 1] * qa_pl[off + v - 1];
  Qp[off] = Qp[off] - s;
}
// rhog -= sum_m flx_h(m)
__global__ void k_update_rho(Dims D, const double *flx, double *rho) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  if (i < D.gmin || i > D.gmax || j < D.gmin || j > D.gmax) return;
  const size_t off = (size_t)kl * D.gall + c, fs = (size_t)D.lall * D.kall * D.gall;
  double s = flx[off];
  for (int m = 1; m < 6; ++m) s = s + flx[m * fs + off];
  rho[off] = rho[off] - s;
}
__global__ void k_update_rho_pl(int kall, const double *flx_pl, double *rho_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const size_t off = (size_t)t * kGallPl;
  double s = flx_pl[off + 1];
  for (int v = 3; v <= 6; ++v) s = s + flx_pl[off + v - 1];
  rho_pl[off] = rho_pl[off] - s;
}

// Thuburn vertical bounds of level k (0-based) of one column, region form (:107-142)
struct VCol {
  const double *q, *ck1, *ck2;
};
__device__ __forceinline__ void vqout(const double *q, const double *ck1, const double *ck2, int k, double &inflagL,
                                      double &Qmin, double &Qmax) {
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  inflagL = 0.5 - sgn(0.5, ck1[k]);
  const double inflagU = 0.5 + sgn(0.5, ck1[k + 1]);
  const double qk = q[k], qm = q[k - 1], qp = q[k + 1];
  const double minL = ((qm < qk) ? qm : qk) + (1.0 - inflagL) * BIG;
  const double minU = ((qp < qk) ? qp : qk) + (1.0 - inflagU) * BIG;
  const double maxL = ((qm > qk) ? qm : qk) - (1.0 - inflagL) * BIG;
  const double maxU = ((qp > qk) ? qp : qk) - (1.0 - inflagU) * BIG;
  double qnmin = (minU < minL) ? minU : minL;
  qnmin = (qk < qnmin) ? qk : qnmin;
  double qnmax = (maxU > maxL) ? maxU : maxL;
  qnmax = (qk > qnmax) ? qk : qnmax;
  const double c1 = ck1[k], c2 = ck2[k];
  const double Cin = inflagL * c1 + inflagU * c2;
  const double Cout = (1.0 - inflagL) * c1 + (1.0 - inflagU) * c2;
  const double CQmin = inflagL * c1 * minL + inflagU * c2 * minU;
  const double CQmax = inflagL * c1 * maxL + inflagU * c2 * maxU;
  const double zerosw = 0.5 - sgn(0.5, fabs(Cout) - EPS);
  const double dv = 0.0;
  Qmin = ((qk - qnmax) + qnmax * (Cin + Cout - dv) - CQmax) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
  Qmax = ((qk - qnmin) + qnmin * (Cin + Cout - dv) - CQmin) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
}

// vertical sub-step of one column (interior columns and the two pole centres)
template <int KMAX>
__global__ void k_vertical(Dims D, int ntr, double dt, double *rho, double *Q, const double *w, double *rho_pl,
                           double *Qp, const double *w_pl, const double *rdgz, const double *afact,
                           const double *bfact) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = D.lall * D.gall;
  double *R, *QQ;
  const double *W;
  size_t s, tstride;
  if (t < ncol) {
    const int l = t / D.gall, c = t % D.gall, G = D.gall_1d;
    const int i = c % G + 1, j = c / G + 1;
    if (i < D.gmin || i > D.gmax || j < D.gmin || j > D.gmax) return;
    const size_t base = (size_t)l * D.kall * D.gall + c;
    R = rho + base, QQ = Q + base, W = w + base, s = D.gall;
    tstride = (size_t)D.lall * D.kall * D.gall;
  } else if (t < ncol + kLallPl) {
    const size_t base = (size_t)(t - ncol) * D.kall * kGallPl;
    R = rho_pl + base, QQ = Qp + base, W = w_pl + base, s = kGallPl;
    tstride = (size_t)kLallPl * D.kall * kGallPl;
  } else {
    return;
  }
  const int K = D.kall, kmin = D.kmin - 1, kmax = D.kmax - 1;  // 0-based
  double ck1[KMAX], ck2[KMAX], q[KMAX], qh[KMAX];
  for (int k = 0; k < K; ++k) ck1[k] = ck2[k] = 0.0;
  for (int k = kmin; k <= kmax; ++k) {
    const double r = R[k * s];
    ck1[k] = -W[k * s] * dt * rdgz[k] / r;
    ck2[k] = W[(k + 1) * s] * dt * rdgz[k] / r;
  }
  ck1[K - 1] = -W[(K - 1) * s] * dt * rdgz[K - 1] / R[(K - 1) * s];
  for (int tr = 0; tr < ntr; ++tr) {
    double *Qt = QQ + tr * tstride;
    for (int k = kmin; k <= kmax; ++k) q[k] = Qt[k * s] / R[k * s];
    q[0] = q[kmin];
    q[K - 1] = q[kmax];
    for (int k = kmin; k <= kmax + 1 && k < K; ++k) qh[k] = afact[k] * q[k] + bfact[k] * q[k - 1];
    // vertical_limiter_thuburn on this column (dyn_vert_adv_limiter/src/mod_src_tracer.f90:107-186)
    double fl, Qmin_km1, Qmax_km1;
    vqout(q, ck1, ck2, kmin, fl, Qmin_km1, Qmax_km1);
    for (int k = kmin + 1; k <= kmax; ++k) {
      double inflagL, Qmin, Qmax;
      vqout(q, ck1, ck2, k, inflagL, Qmin, Qmax);
      const double h = qh[k];
      const double a1 = (h < Qmax_km1) ? h : Qmax_km1;
      const double b1 = (Qmin_km1 > a1) ? Qmin_km1 : a1;
      const double a2 = (h < Qmax) ? h : Qmax;
      const double b2 = (Qmin > a2) ? Qmin : a2;
      qh[k] = inflagL * b1 + (1.0 - inflagL) * b2;
      Qmin_km1 = Qmin;
      Qmax_km1 = Qmax;
    }
    for (int k = kmin; k <= kmax; ++k) {
      const double fu = W[(k + 1) * s] * qh[k + 1], flo = W[k * s] * qh[k];
      Qt[k * s] = Qt[k * s] - (fu - flo) * dt * rdgz[k];
    }
    Qt[0] = Qt[kmin * s];
    Qt[(K - 1) * s] = Qt[kmax * s];
  }
  for (int k = kmin; k <= kmax; ++k) R[k * s] = R[k * s] - (W[(k + 1) * s] - W[k * s]) * dt * rdgz[k];
  R[0] = R[kmin * s];
  R[(K - 1) * s] = R[kmax * s];
}

// ---------------------------------------------------------------------------
static dim3 slab(const Dims &D, int th) { return dim3((D.gall + th - 1) / th, D.kall * D.lall); }
static constexpr int kSlabThreads = 128;

static size_t n3_of(const Dims &D) { return (size_t)D.gall * D.kall * D.lall; }
static size_t n3p_of(const Dims &D) { return (size_t)kGallPl * D.kall * kLallPl; }

void launch_courant(const StepCtx &S, const double *rhog, const double *rhog_pl, cudaStream_t st) {
  const size_t n3 = n3_of(S.D), n3p = n3p_of(S.D);
  k_courant<<<(unsigned)((6 * n3 + 255) / 256), 256, 0, st>>>((int)n3, S.flx, rhog, S.ch, S.cm);
  k_courant_pl<<<(unsigned)((n3p + 255) / 256), 256, 0, st>>>(S.D.kall, S.flx_pl, rhog_pl, S.ch_pl, S.cm_pl);
}

void launch_divide(const StepCtx &S, const double *Q, const double *Qp, const double *rhog, const double *rhog_pl,
                   cudaStream_t st) {
  const size_t n3 = n3_of(S.D), n3p = n3p_of(S.D);
  k_divide<<<(unsigned)((n3 + n3p + 255) / 256), 256, 0, st>>>((long long)n3, (int)n3p, Q, rhog, Qp, rhog_pl, S.q,
                                                               S.q_pl);
}

void launch_gradient(const StepCtx &S, cudaStream_t st) {
  const Dims &D = S.D;
  k_gradient<<<slab(D, kSlabThreads), kSlabThreads, 0, st>>>(D, S.q, S.cg, S.grad);
  k_gradient_pl<<<(unsigned)((kLallPl * D.kall + 255) / 256), 256, 0, st>>>(D.kall, S.q_pl, S.cg_pl, S.grad_pl);
  launch_gather<double>(D, S.plan.n, S.plan.dst, S.plan.src, D.kall, 3, S.grad, S.grad_pl, st);
}

void launch_remap(const StepCtx &S, cudaStream_t st) {
  const Dims &D = S.D;
  k_remap<<<slab(D, kSlabThreads), kSlabThreads, 0, st>>>(D, S.q, S.grad, S.cm, S.xc, S.GRD_x, S.qa);
  k_remap_pl<<<(unsigned)((n3p_of(D) + 255) / 256), 256, 0, st>>>(D.kall, S.q_pl, S.grad_pl, S.cm_pl, S.xc_pl,
                                                                   S.GRD_x_pl, S.qa_pl);
}

void launch_update_h(const StepCtx &S, const double *qa, const double *qa_pl, double *Q, double *Qp, cudaStream_t st) {
  const Dims &D = S.D;
  k_update_h<<<slab(D, kSlabThreads), kSlabThreads, 0, st>>>(D, S.flx, qa, Q);
  k_update_h_pl<<<(unsigned)((kLallPl * D.kall + 255) / 256), 256, 0, st>>>(D.kall, S.flx_pl, qa_pl, Qp);
}

void launch_update_rho(const StepCtx &S, double *rho, double *rho_pl, cudaStream_t st) {
  const Dims &D = S.D;
  k_update_rho<<<slab(D, kSlabThreads), kSlabThreads, 0, st>>>(D, S.flx, rho);
  k_update_rho_pl<<<(unsigned)((kLallPl * D.kall + 255) / 256), 256, 0, st>>>(D.kall, S.flx_pl, rho_pl);
}

int step_plain(StepCtx &S, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
               const double *vx, const double *vx_pl, const double *vy, const double *vy_pl, const double *vz,
               const double *vz_pl, const double *w, const double *w_pl, cudaStream_t st, long long &launches) {
  const Dims &D = S.D;
  const size_t n3 = n3_of(D), n3p = n3p_of(D);
  // shared per step
  FluxIn<double> fin{rhog, rhog_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl};
  FluxOut<double> fout{S.flx, S.flx_pl, S.xc, S.xc_pl};
  launch_horizontal_flux<double>(D, fin, fout, S.geo, dt, st);
  launch_courant(S, rhog, rhog_pl, st);
  launches += 4;
  LimIn<double> lin{S.q, S.q_pl, S.zero, S.zero_pl, S.ch, S.ch_pl, S.cm, S.cm_pl};
  for (int t = 0; t < ntr; ++t) {
    double *Q = rhogq + t * n3, *Qp = rhogq_pl + t * n3p;
    launch_divide(S, Q, Qp, rhog, rhog_pl, st);
    launch_gradient(S, st);
    launch_remap(S, st);
    launch_hlim_qout<double>(D, lin, S.qout, S.qout_pl, S.qin_pl, st);
    launch_gather<double>(D, S.plan.n, S.plan.dst, S.plan.src, D.kall, 2, S.qout, S.qout_pl, st);
    launch_hlim_apply<double>(D, lin, S.qa, S.qa_pl, S.qout, S.qout_pl, S.qin_pl, st);
    launch_update_h(S, S.qa, S.qa_pl, Q, Qp, st);
    launches += 14;
  }
  launch_update_rho(S, rhog, rhog_pl, st);
  const int ncol = D.lall * D.gall + kLallPl;
  if (D.kall <= 48)
    k_vertical<48><<<(ncol + 127) / 128, 128, 0, st>>>(D, ntr, dt, rhog, rhogq, w, rhog_pl, rhogq_pl, w_pl, S.rdgz,
                                                       S.afact, S.bfact);
  else if (D.kall <= 128)
    k_vertical<128><<<(ncol + 127) / 128, 128, 0, st>>>(D, ntr, dt, rhog, rhogq, w, rhog_pl, rhogq_pl, w_pl, S.rdgz,
                                                        S.afact, S.bfact);
  else
    return ICA_ERR_ARG;
  launch_gather<double>(D, S.plan.n, S.plan.dst, S.plan.src, D.kall, 1, rhog, rhog_pl, st);
  launch_gather<double>(D, S.plan.n, S.plan.dst, S.plan.src, D.kall, ntr, rhogq, rhogq_pl, st);
  launches += 5;
  return ICA_OK;
}

}  // namespace icoadv
