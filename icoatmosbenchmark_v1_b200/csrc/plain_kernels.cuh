// Launch interface of the plain kernels (one kernel per reference subroutine).
#pragma once

#include <cuda_runtime.h>

#include "icoadv_internal.h"

namespace icoadv {

// Fortran parameter indices of problem_size.inc:14-20,95-104,122
enum : int { TI = 1, TJ = 2 };
enum : int { AI = 1, AIJ = 2, AJ = 3 };
enum : int { W1 = 3, W2 = 4, W3 = 5 };
enum : int { HNX = 1, HNY = 2, HNZ = 3 };
enum : int { P_RAREA = 2 };

// Sizes as seen by the kernels (ADM_* of problem_size.inc:28-59).
struct Dims {
  int gall_1d, gall, gmin, gmax;  // 1-based gmin/gmax
  int kall, kmin, kmax;           // 1-based kmin/kmax
  int lall;
  const int *have_sgp;            // device array [lall]
  int have_pl;                    // ADM_have_pl: the pole regions are processed
};

template <typename T> struct Geo {
  const T *GRD_xr, *GRD_xr_pl, *GMTR_p, *GMTR_p_pl, *GMTR_t, *GMTR_t_pl, *GMTR_a, *GMTR_a_pl;
};
template <typename T> struct FluxIn {
  const T *rho, *rho_pl, *rhovx, *rhovx_pl, *rhovy, *rhovy_pl, *rhovz, *rhovz_pl;
};
template <typename T> struct FluxOut {
  T *flx_h, *flx_h_pl, *GRD_xc, *GRD_xc_pl;
};
template <typename T> struct LimIn {
  const T *q, *q_pl, *d, *d_pl, *ch, *ch_pl, *cmask, *cmask_pl;
};

template <typename T>
void launch_horizontal_flux(const Dims &D, const FluxIn<T> &in, const FluxOut<T> &out, const Geo<T> &g, T dt,
                            cudaStream_t s);
// Qout (pre-fill) for regions and poles; Qin_pl(6,kall,2,2,2) is kept for the apply
template <typename T>
void launch_hlim_qout(const Dims &D, const LimIn<T> &in, T *Qout, T *Qout_pl, T *Qin_pl, cudaStream_t s);
template <typename T>
void launch_hlim_apply(const Dims &D, const LimIn<T> &in, T *q_a, T *q_a_pl, const T *Qout, const T *Qout_pl,
                       const T *Qin_pl, cudaStream_t s);
template <typename T>
void launch_vlim(const Dims &D, T *q_h, T *q_h_pl, const T *q, const T *q_pl, const T *d, const T *d_pl,
                 const T *ck, const T *ck_pl, cudaStream_t s);
template <typename T>
void launch_gather(const Dims &D, int nent, const int *dst, const int *src, int kmax, int vmax, T *var, T *var_pl,
                   cudaStream_t s);

}  // namespace icoadv
