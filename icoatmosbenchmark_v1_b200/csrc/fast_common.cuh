// Shared device code of the batched path: one instance of the grid, the FP64
// face geometry and face bounds with every special case of the reference
// (singular point, index clamps, unused faces), usable on global or shared data.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cfloat>

#include "plain_kernels.cuh"

namespace icoadv {

// One grid instance of the batched path (device pointers; region arrays in the
// reference layout (m, lall, kall, gall), pole arrays (m, 2, kall, 6)).
struct FastInst {
  int G, gall, gmin, gmax, K, kmin, kmax, lall, ntr, ntx, nty;  // ntx/nty: tiles per region side
  double dt;
  const int *have_sgp;
  const double *GMTR_p, *GMTR_t, *GMTR_a, *GRD_xr, *GRD_x, *cg;
  const double *GMTR_p_pl, *GMTR_t_pl, *GMTR_a_pl, *GRD_xr_pl, *GRD_x_pl, *cg_pl;
  const float *cg32;   // coef_grad in FP32, (lall, 3, 7, gall)
  // remap offsets GRD_xr - GRD_x per face, FP32, (lall, 18, gall), followed by the face
  // geometry of each column, (lall, 16, gall): TI W1..W3, TJ W1..W3, HN x/y/z of the faces
  // AI, AIJ, AJ, rarea (fast_face_geo)
  const float *off32;
  const double *rdgz, *afact, *bfact;
  // fields: FP32 (the FP32 variant) or, when f64 is set, FP64 (the FP64 variant: every face
  // value, bound and limiter in FP64, so the batched step follows the plain FP64 step)
  int f64;
  const float *vx, *vy, *vz, *w, *vx_pl, *vy_pl, *vz_pl, *w_pl;
  const double *vx64, *vy64, *vz64, *w64, *vx64_pl, *vy64_pl, *vz64_pl, *w64_pl;
  const double *off64;  // remap offsets in FP64 (FP64 variant), layout of off32
  const double *rho_in, *rho_in_pl, *Q_in, *Q_in_pl;
  double *rho_out, *rho_out_pl, *Q_out, *Q_out_pl;
  // region-boundary / pole values of grad and Qout, computed once per step
  const int *bsrc;   // (lall, gall): -1 interior non-boundary, >= 0 boundary index, -2 halo without source
  const int *blist;  // (nb): point index of boundary entry b (region cell, or pole centre when >= lall*gall)
  const int *pole_ring_b;  // (2, 5): boundary index feeding pole ring slot v = 2..6
  int nb;
  const int *carry;  // (ncarry): region points no halo list writes; they keep their input values
  int ncarry;
  // faces with a halo cell on one side ("seam" faces), precomputed in FP64 each step
  const int *seam_list;  // (ns): (l*gall + owner cell)*3 + face (0..2)
  const int *seam_id;    // (lall, gall, 3): index into seam_list, -1 for faces between interior cells
  int ns;
  double *sflux;  // (K, ns): 0.5 (rhov . HN) of the seam faces
  float *sval;    // (ntr, K, ns): limited face values of the seam faces
  double *sval64;  // the same in FP64 (FP64 variant)
  double *bbuf;  // (ntr, K, nb, 5): grad x, y, z, Qout min, Qout max
  double *Fg;    // (3, lall, K, gall): face flux 0.5 (rhov . HN) of the 3 faces of each owner, per step
  // (3, lall, K, gall) per owner face a: x, y, z = GRD_xc - GRD_x of the face's upwind cell (the
  // remap displacement that cell applies to its gradient); w = the owner-side upwind mask of
  // horizontal_limiter_thuburn (1: the neighbour is upwind, 0: the owner is)
  float4 *dupc;
  float4 *vco;   // (lall, K, gall): ck(k,1), ck(k,2), 1/rhog, rhogw(k) after the horizontal sub-step
  double4 *vco64;  // the same in FP64 (FP64 variant)
  double4 *dupc64;  // dupc in FP64 (FP64 variant)
  unsigned long long *work_next;  // work-item counter of the persistent horizontal kernel
  int *err;  // device status word: bit 0 = a bounded wait of the horizontal kernel gave up
  // the regions [l0, l1) this instance computes (a rank of a region-sharded run; the whole
  // grid otherwise), and whether it computes the two pole centres
  int l0, l1, poles;
};

// Planes of the per-column tables that follow the remap offsets (see FastInst::off32).
constexpr int kOffPlanes = 18, kFaceGeoPlanes = 16;
template <typename T>
__device__ __forceinline__ const T *fast_face_geo(const T *off, const FastInst &I) {
  return off + (size_t)I.lall * kOffPlanes * I.gall;
}

// Is point p (region point l*gall + ij, or a pole point after them) computed by instance I?
__device__ __forceinline__ bool owns_point(const FastInst &I, int p) {
  if (p >= I.lall * I.gall) return I.poles != 0;
  const int l = p / I.gall;
  return l >= I.l0 && l < I.l1;
}

// TMA descriptors of one instance's tile windows (built on the host per step, since the state
// buffers alternate): rhogq_in as (i, j, l*K + k, tracer) FP64 and rhog_in as (i, j, l*K + k).
struct TileMaps {
  CUtensorMap q, rho;
};

// Up to kMaxInst grid instances advanced by the same launches (batches of uneven grid
// levels); passed by value as a __grid_constant__ kernel parameter.
constexpr int kMaxInst = 4;
struct MultiInst {
  int n;
  FastInst inst[kMaxInst];
};
struct MultiMaps {
  TileMaps m[kMaxInst];
};

// Instance of flat work item w, given the number of work items cnt(inst) of each
// instance; w becomes the index within that instance.  -1 when w is past the end.
template <class F>
__device__ __forceinline__ int find_inst(const MultiInst &M, long long &w, F cnt) {
  for (int i = 0; i < M.n; ++i) {
    const long long c = cnt(M.inst[i]);
    if (w < c) return i;
    w -= c;
  }
  return -1;
}

__device__ __forceinline__ double fsg(double a, double b) { return copysign(fabs(a), b); }
__device__ __forceinline__ double mn64(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double mx64(double a, double b) { return (b > a) ? b : a; }
// FP32 min / max: one FMNMX instruction each (the select form takes a compare and a select).
// Operands here are never NaN; for them the two agree except for the sign of a zero result.
__device__ __forceinline__ float mn32(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float mx32(float a, float b) { return fmaxf(a, b); }

// field readers at flat offset o: var 0..3 = rhogvx, rhogvy, rhogvz, rhogw (FP64 of either variant)
__device__ __forceinline__ double fld(const FastInst &I, int var, size_t o) {
  if (I.f64) return (var == 0 ? I.vx64 : var == 1 ? I.vy64 : var == 2 ? I.vz64 : I.w64)[o];
  return (double)(var == 0 ? I.vx : var == 1 ? I.vy : var == 2 ? I.vz : I.w)[o];
}
__device__ __forceinline__ double fld_pl(const FastInst &I, int var, size_t o) {
  if (I.f64) return (var == 0 ? I.vx64_pl : var == 1 ? I.vy64_pl : var == 2 ? I.vz64_pl : I.w64_pl)[o];
  return (double)(var == 0 ? I.vx_pl : var == 1 ? I.vy_pl : var == 2 ? I.vz_pl : I.w_pl)[o];
}

// arithmetic of the tile and column kernels: FP32 (float) or FP64 (double)
template <typename R> struct Arith;
template <> struct Arith<float> {
  using V2 = float2;
  using V4 = float4;
  static constexpr float BIG = FLT_MAX, RR_EPS = FLT_EPSILON;
  static __device__ __forceinline__ float mn(float a, float b) { return fminf(a, b); }
  static __device__ __forceinline__ float mx(float a, float b) { return fmaxf(a, b); }
  static __device__ __forceinline__ float sgn(float a, float b) { return copysignf(a, b); }
  static __device__ __forceinline__ V2 v2(float a, float b) { return make_float2(a, b); }
};
template <> struct Arith<double> {
  using V2 = double2;
  using V4 = double4;
  static constexpr double BIG = DBL_MAX, RR_EPS = DBL_EPSILON;
  static __device__ __forceinline__ double mn(double a, double b) { return (b < a) ? b : a; }
  static __device__ __forceinline__ double mx(double a, double b) { return (b > a) ? b : a; }
  static __device__ __forceinline__ double sgn(double a, double b) { return copysign(a, b); }
  static __device__ __forceinline__ V2 v2(double a, double b) { return make_double2(a, b); }
};

// geometry readers (region coords i,j 1-based)
__device__ __forceinline__ double gt(const FastInst &I, int l, int i, int j, int t, int w) {
  return I.GMTR_t[((size_t)(w - 1) * 2 + (t - 1)) * I.lall * I.gall + (size_t)l * I.gall + (j - 1) * I.G + (i - 1)];
}
__device__ __forceinline__ double ga(const FastInst &I, int l, int i, int j, int a, int h) {
  return I.GMTR_a[((size_t)(h - 1) * 3 + (a - 1)) * I.lall * I.gall + (size_t)l * I.gall + (j - 1) * I.G + (i - 1)];
}
__device__ __forceinline__ double gxr(const FastInst &I, int l, int i, int j, int a, int x) {
  return I.GRD_xr[((size_t)(x - 1) * 3 + (a - 1)) * I.lall * I.gall + (size_t)l * I.gall + (j - 1) * I.G + (i - 1)];
}
__device__ __forceinline__ double rarea(const FastInst &I, int l, int i, int j) {
  return I.GMTR_p[(size_t)(P_RAREA - 1) * I.lall * I.gall + (size_t)l * I.gall + (j - 1) * I.G + (i - 1)];
}
__device__ __forceinline__ double gx(const FastInst &I, int l, int i, int j, int x) {
  return I.GRD_x[(size_t)x * I.lall * I.gall + (size_t)l * I.gall + (j - 1) * I.G + (i - 1)];
}

struct T4 {
  double r, x, y, z;
};

// Triangle-vertex values (rho, rhov) of dyn_horiz_adv_flux/src/mod_src_tracer.f90:141-201.
// Acc: double operator()(int var, int i, int j) with var 0 = rho, 1..3 = rhovx..z.
template <class Acc>
__device__ __forceinline__ T4 triTI(const FastInst &I, int l, int i, int j, const Acc &f) {
  const double w1 = gt(I, l, i, j, TI, W1), w2 = gt(I, l, i, j, TI, W2), w3 = gt(I, l, i, j, TI, W3);
  T4 t;
  t.r = f(0, i, j) * w1 + f(0, i + 1, j) * w2;
  t.x = f(1, i, j) * w1 + f(1, i + 1, j) * w2;
  t.y = f(2, i, j) * w1 + f(2, i + 1, j) * w2;
  t.z = f(3, i, j) * w1 + f(3, i + 1, j) * w2;
  t.r = t.r + f(0, i + 1, j + 1) * w3;
  t.x = t.x + f(1, i + 1, j + 1) * w3;
  t.y = t.y + f(2, i + 1, j + 1) * w3;
  t.z = t.z + f(3, i + 1, j + 1) * w3;
  return t;
}
template <class Acc>
__device__ __forceinline__ T4 triTJ(const FastInst &I, int l, int i, int j, const Acc &f) {
  const double w1 = gt(I, l, i, j, TJ, W1), w2 = gt(I, l, i, j, TJ, W2), w3 = gt(I, l, i, j, TJ, W3);
  T4 t;
  t.r = f(0, i, j) * w1;
  t.x = f(1, i, j) * w1;
  t.y = f(2, i, j) * w1;
  t.z = f(3, i, j) * w1;
  t.r = t.r + f(0, i + 1, j + 1) * w2 + f(0, i, j + 1) * w3;
  t.x = t.x + f(1, i + 1, j + 1) * w2 + f(1, i, j + 1) * w3;
  t.y = t.y + f(2, i + 1, j + 1) * w2 + f(2, i, j + 1) * w3;
  t.z = t.z + f(3, i + 1, j + 1) * w2 + f(3, i, j + 1) * w3;
  return t;
}
template <class Acc>
__device__ __forceinline__ T4 triTIs(const FastInst &I, int l, int i, int j, bool sgp, const Acc &f) {
  if (sgp && i == I.gmin - 1 && j == I.gmin - 1) return triTJ(I, l, i + 1, j, f);
  return triTI(I, l, i, j, f);
}

// Does face a of owner (i,j) exist in horizontal_flux's loops (:235-309)?
__device__ __forceinline__ bool face_exists(const FastInst &I, int i, int j, int a) {
  const int g0 = I.gmin, g1 = I.gmax;
  if (a == AI) return j >= g0 && j <= g1 && i >= g0 - 1 && i <= g1;
  if (a == AIJ) return i >= g0 - 1 && i <= g1 && j >= g0 - 1 && j <= g1;
  return i >= g0 && i <= g1 && j >= g0 - 1 && j <= g1;
}

// flux = 0.5 (rhov . HN) of face a of owner (i,j) and the mass centroid GRD_xc, FP64.
template <class Acc>
__device__ __forceinline__ double face_geo(const FastInst &I, int l, int i, int j, int a, bool sgp, const Acc &f,
                                           double xc[3]) {
  T4 p, q;
  if (a == AI) {
    p = triTJ(I, l, i, j - 1, f);
    q = triTIs(I, l, i, j, sgp, f);
  } else if (a == AIJ) {
    p = triTIs(I, l, i, j, sgp, f);
    q = triTJ(I, l, i, j, f);
  } else {
    p = triTJ(I, l, i, j, f);
    q = triTIs(I, l, i - 1, j, sgp, f);
  }
  const double rr = 1.0 / mx64(p.r + q.r, DBL_EPSILON);
  const double vx = p.x + q.x, vy = p.y + q.y, vz = p.z + q.z;
  const double flux = 0.5 * (vx * ga(I, l, i, j, a, HNX) + vy * ga(I, l, i, j, a, HNY) + vz * ga(I, l, i, j, a, HNZ));
  xc[0] = gxr(I, l, i, j, a, 1) - vx * rr * I.dt * 0.5;
  xc[1] = gxr(I, l, i, j, a, 2) - vy * rr * I.dt * 0.5;
  xc[2] = gxr(I, l, i, j, a, 3) - vz * rr * I.dt * 0.5;
  return flux;
}

// 4-point bounds of face a of cell (i,j) incl. the clamps (:152-153) and the singular AIJ stencil (:192-214)
template <class QAcc>
__device__ __forceinline__ void bounds64(const FastInst &I, int i, int j, int a, bool sgp, const QAcc &q,
                                         double &lo, double &hi) {
  const int G = I.G;
  const int ij = (j - 1) * G + i;
  int im1j = ij - 1, ijm1 = ij - G;
  if (im1j < 1) im1j = 1;
  if (ijm1 < 1) ijm1 = 1;
  auto Q = [&](int cell) { return q((cell - 1) % G + 1, (cell - 1) / G + 1); };
  const double q0 = Q(ij);
  double b, c, d;
  if (a == AI) {
    b = Q(ijm1), c = Q(ij + 1), d = Q(ij + G + 1);
  } else if (a == AIJ) {
    if (sgp && i == I.gmin - 1 && j == I.gmin - 1) b = Q(ij + G + 1), c = Q(ij + G + 2), d = Q(ij + G);
    else b = Q(ij + 1), c = Q(ij + G + 1), d = Q(ij + G);
  } else {
    b = Q(ij + G + 1), c = Q(ij + G), d = Q(im1j);
  }
  lo = mn64(mn64(mn64(q0, b), c), d);
  hi = mx64(mx64(mx64(q0, b), c), d);
}

// flx_h(c, m) of the reference from face fluxes (FP64), with halo zeros and the singular zero
__device__ __forceinline__ double cell_flx(const FastInst &I, int l, int i, int j, int m, bool sgp, double flux_of_face,
                                           double ra) {
  if (m <= 3) return flux_of_face * ra * I.dt;
  if (m == 6 && sgp && i == I.gmin && j == I.gmin) return 0.0;
  return -flux_of_face * ra * I.dt;
}

}  // namespace icoadv
