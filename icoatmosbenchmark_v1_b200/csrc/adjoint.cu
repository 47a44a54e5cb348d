// Reverse mode (adjoint) of the composed FP64 step of step.cu.
//
// Given the step's input state (a checkpoint) and the adjoint of its output,
// the forward intermediates are recomputed with the step's own kernels, then
// every operation is transposed in reverse order: the final halo fill, the
// vertical sub-step (column by column), the horizontal rhogq update, the
// limiter apply and the Qout halo fill, the Qout bounds, the upwind remap,
// the gradient and its halo fill, q = rhogq / rhog, the density update, the
// Courant numbers and horizontal_flux (dyn_horiz_adv_flux/src/
// mod_src_tracer.f90:42-379), whose triangle interpolation carries the
// adjoint to rhog and the three wind components.
//
// Kinks follow the forward's own comparisons (subgradients, as in
// tangent-linear models): min/max pass the adjoint to the operand the forward
// returned (the first one on a tie), a clamp to its input when the input was
// returned and to the binding bound otherwise; the upwind masks, inflow flags
// and zero-outflow switches are held fixed; terms that carry +-BIG (the
// outflow side of a masked bound) have no derivative.  rhogw, the geometry
// and the vertical grid are constants.
//
// Transposes of scatter shape (a face handing its adjoint to the cell that
// bounded it, a halo copy handing its adjoint to the source point) use FP64
// atomicAdd; the gradient stencil and the triangle interpolation are
// transposed as gathers.  Sums therefore associate differently from a serial
// adjoint, at rounding level.
#include <cuda_runtime.h>

#include <cfloat>

#include "adjoint.cuh"

namespace icoadv {

namespace {

constexpr double kEps = DBL_EPSILON, kBig = DBL_MAX;

__device__ __forceinline__ double mn(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double mx(double a, double b) { return (b > a) ? b : a; }
__device__ __forceinline__ double sgn(double a, double b) { return copysign(fabs(a), b); }

// which operand of mn(mn(mn(a,b),c),d) / the mx chain is returned (0..3)
__device__ __forceinline__ int argmin4(const double v[4]) {
  int i = 0;
  double s = v[0];
  if (v[1] < s) s = v[1], i = 1;
  if (v[2] < s) s = v[2], i = 2;
  if (v[3] < s) i = 3;
  return i;
}
__device__ __forceinline__ int argmax4(const double v[4]) {
  int i = 0;
  double s = v[0];
  if (v[1] > s) s = v[1], i = 1;
  if (v[2] > s) s = v[2], i = 2;
  if (v[3] > s) i = 3;
  return i;
}

__device__ __forceinline__ bool inner(const Dims &D, int i, int j) {
  return i >= D.gmin && i <= D.gmax && j >= D.gmin && j <= D.gmax;
}

// The 4 cells (0-based slab indices) bounding face a (1..3) of owner (i,j): the owner
// first, with the index clamps and the singular AIJ stencil of the limiter
// (dyn_horiz_adv_limiter/src/mod_src_tracer.f90:152-214).
__device__ __forceinline__ void face_points(const Dims &D, int i, int j, int a, bool sgp, int p[4]) {
  const int G = D.gall_1d, ij = (j - 1) * G + i;
  int im1j = ij - 1, ijm1 = ij - G;
  if (im1j < 1) im1j = 1;
  if (ijm1 < 1) ijm1 = 1;
  p[0] = ij - 1;
  if (a == 1) {
    p[1] = ijm1 - 1, p[2] = ij, p[3] = ij + G;
  } else if (a == 2) {
    if (sgp && i == D.gmin - 1 && j == D.gmin - 1) p[1] = ij + G, p[2] = ij + G + 1, p[3] = ij + G - 1;
    else p[1] = ij, p[2] = ij + G, p[3] = ij + G - 1;
  } else {
    p[1] = ij + G, p[2] = ij + G - 1, p[3] = im1j - 1;
  }
}

// ---------------------------------------------------------------------------
// halo fill: every copied point hands its adjoint to its source and drops it
// (the composed plan never reads a point it writes)
__global__ void k_fill_adj(int nent, const int *__restrict__ dst, const int *__restrict__ src, int npt_rgn,
                           int gall, int lall, int kmax, int vmax, double *a, double *a_pl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nent * kmax * vmax) return;
  const int e = (int)(t % nent), kv = (int)(t / nent), k = kv % kmax, v = kv / kmax;
  auto addr = [&](int p) -> double * {
    if (p < npt_rgn) return a + (((size_t)v * lall + p / gall) * kmax + k) * gall + p % gall;
    const int qd = p - npt_rgn;
    return a_pl + (((size_t)v * kLallPl + qd / kGallPl) * kmax + k) * kGallPl + qd % kGallPl;
  };
  double *pd = addr(dst[e]);
  const double x = *pd;
  if (x == 0.0) return;
  *pd = 0.0;
  atomicAdd(addr(src[e]), x);
}

// ---------------------------------------------------------------------------
// vertical sub-step, density part: rhog(kall) = rhog(kmax), rhog(1) = rhog(kmin),
// rhog(k) = rho_h(k) - d(rhogw)/dz dt.  The adjoint of rho_h goes to a_rh; the
// input adjoint (a_rho in place) keeps what passes through the step unchanged
// (halo columns, pole ring points) and is zero elsewhere so far.
__global__ void k_adj_vrho(Dims D, double *a_rho, double *a_rho_pl, double *a_rh, double *a_rh_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = D.lall * D.gall;
  double *aR, *aH;
  size_t s;
  bool col;
  if (t < ncol) {
    const int l = t / D.gall, c = t % D.gall, G = D.gall_1d;
    const size_t base = (size_t)l * D.kall * D.gall + c;
    aR = a_rho + base, aH = a_rh + base, s = D.gall;
    col = inner(D, c % G + 1, c / G + 1);
  } else if (t < ncol + kLallPl * kGallPl) {
    const int p = t - ncol, l = p / kGallPl, v = p % kGallPl;
    const size_t base = (size_t)l * D.kall * kGallPl + v;
    aR = a_rho_pl + base, aH = a_rh_pl + base, s = kGallPl;
    col = (v == 0);
  } else {
    return;
  }
  const int K = D.kall, kmin = D.kmin - 1, kmax = D.kmax - 1;  // 0-based
  if (!col) {
    for (int k = 0; k < K; ++k) aH[k * s] = 0.0;
    return;
  }
  aR[kmax * s] += aR[(K - 1) * s];
  aR[(K - 1) * s] = 0.0;
  aR[kmin * s] += aR[0];
  aR[0] = 0.0;
  for (int k = 0; k < K; ++k) {
    aH[k * s] = (k >= kmin && k <= kmax) ? aR[k * s] : 0.0;
    aR[k * s] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// vertical sub-step of one tracer, one column per thread, levels streamed from the top.
//
// Forward (step.cu k_vertical, mod_src_tracer.f90:107-186 with d = 0):
//   qc(k) = Qh(k) / rh(k), ghosts qc(1) = qc(kmin), qc(kall) = qc(kmax)
//   ck1(k) = -w(k) dt rdgz(k) / rh(k), ck2(k) = w(k+1) dt rdgz(k) / rh(k), ck1(kall) likewise
//   qh(k) = afact(k) qc(k) + bfact(k) qc(k-1), clamped to the Qout bounds of level k-1 or k
//   Q(k) = Qh(k) - (w(k+1) qh(k+1) - w(k) qh(k)) dt rdgz(k), ghosts copied
// The column adjoint's per-level inputs stream through a shared-memory ring of kAdjStages
// levels, filled by each thread's own cp.async copies (no barrier: a thread reads only what it
// copied), so kAdjStages - 1 levels of a column are in flight while a level is worked on
// (a 4-step sweep at gl7, 4 tracers: 124.2 -> 118.5 ms against plain loads of each level).
constexpr int kAdjStages = 4, kAdjThreads = 128;
struct AdjRing {
  double v[kAdjStages][6][kAdjThreads];  // Qh(kk), rh(kk), rh(k), w(k), w(k+1), aQ(k)
};
__device__ __forceinline__ unsigned adj_smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void adj_cp8(double *dst, const double *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(adj_smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void adj_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void adj_drain() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void adj_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

struct VLev {  // one level's inputs
  double qc, R, w, c1, c2, aO;
};
struct VLim {  // one level's Thuburn bounds and what they were made of
  double infL, infU, c1, c2, mnL, mnU, mxL, mxU, qnmin, qnmax, Cin, Cout, zsw, Qmn, Qmx;
  int amin, amax;
};

__device__ __forceinline__ VLim vlim_level(double qm, double qk, double qp, double c1, double c1u, double c2) {
  VLim v;
  v.infL = 0.5 - sgn(0.5, c1);
  v.infU = 0.5 + sgn(0.5, c1u);
  v.c1 = c1, v.c2 = c2;
  v.mnL = mn(qk, qm) + (1.0 - v.infL) * kBig;
  v.mnU = mn(qk, qp) + (1.0 - v.infU) * kBig;
  v.mxL = mx(qk, qm) - (1.0 - v.infL) * kBig;
  v.mxU = mx(qk, qp) - (1.0 - v.infU) * kBig;
  const double t1 = mn(v.mnL, v.mnU);
  v.qnmin = mn(t1, qk);
  v.amin = (qk < t1) ? 2 : ((v.mnU < v.mnL) ? 1 : 0);
  const double t2 = mx(v.mxL, v.mxU);
  v.qnmax = mx(t2, qk);
  v.amax = (qk > t2) ? 2 : ((v.mxU > v.mxL) ? 1 : 0);
  v.Cin = v.infL * c1 + v.infU * c2;
  v.Cout = (1.0 - v.infL) * c1 + (1.0 - v.infU) * c2;
  const double CQmin = v.infL * c1 * v.mnL + v.infU * c2 * v.mnU;
  const double CQmax = v.infL * c1 * v.mxL + v.infU * c2 * v.mxU;
  v.zsw = 0.5 - sgn(0.5, fabs(v.Cout) - kEps);
  v.Qmn = ((qk - v.qnmax) + v.qnmax * (v.Cin + v.Cout) - CQmax) / (v.Cout + v.zsw) * (1.0 - v.zsw) + qk * v.zsw;
  v.Qmx = ((qk - v.qnmin) + v.qnmin * (v.Cin + v.Cout) - CQmin) / (v.Cout + v.zsw) * (1.0 - v.zsw) + qk * v.zsw;
  return v;
}

// adjoint of (Qout_min, Qout_max) of one level -> qc(k-1), qc(k), qc(k+1), ck1(k), ck2(k)
__device__ __forceinline__ void vlim_level_adj(const VLim &v, double qm, double qk, double qp, double aQm,
                                               double aQx, double &am, double &a0, double &ap, double &ac1,
                                               double &ac2) {
  if (aQm == 0.0 && aQx == 0.0) return;
  if (v.zsw != 0.0) {
    a0 += aQm + aQx;
    return;
  }
  const double c1 = v.c1, c2 = v.c2;
  const double Dn = v.Cout, S = v.Cin + v.Cout;
  const double CQmax = v.infL * c1 * v.mxL + v.infU * c2 * v.mxU;
  const double CQmin = v.infL * c1 * v.mnL + v.infU * c2 * v.mnU;
  const double Nmn = (qk - v.qnmax) + v.qnmax * S - CQmax, Nmx = (qk - v.qnmin) + v.qnmin * S - CQmin;
  const double rD = 1.0 / Dn;
  const double aNmn = aQm * rD, aNmx = aQx * rD;
  const double aD = -(aNmn * Nmn + aNmx * Nmx) * rD;
  double a_qk = aNmn + aNmx;
  const double a_qnmax = aNmn * (S - 1.0), a_qnmin = aNmx * (S - 1.0);
  const double aS = aNmn * v.qnmax + aNmx * v.qnmin;
  const double aCQmax = -aNmn, aCQmin = -aNmx;
  const double aCin = aS, aCout = aS + aD;
  double amxL = aCQmax * v.infL * c1, amxU = aCQmax * v.infU * c2;
  double amnL = aCQmin * v.infL * c1, amnU = aCQmin * v.infU * c2;
  double a1 = aCin * v.infL + aCout * (1.0 - v.infL);
  double a2 = aCin * v.infU + aCout * (1.0 - v.infU);
  if (v.infL != 0.0) a1 += aCQmax * v.infL * v.mxL + aCQmin * v.infL * v.mnL;
  if (v.infU != 0.0) a2 += aCQmax * v.infU * v.mxU + aCQmin * v.infU * v.mnU;
  if (v.amax == 2) a_qk += a_qnmax;
  else if (v.amax == 1) amxU += a_qnmax;
  else amxL += a_qnmax;
  if (v.amin == 2) a_qk += a_qnmin;
  else if (v.amin == 1) amnU += a_qnmin;
  else amnL += a_qnmin;
  if (v.infL != 0.0) {
    if (qm < qk) am += amnL;
    else a_qk += amnL;
    if (qm > qk) am += amxL;
    else a_qk += amxL;
  }
  if (v.infU != 0.0) {
    if (qp < qk) ap += amnU;
    else a_qk += amnU;
    if (qp > qk) ap += amxU;
    else a_qk += amxU;
  }
  a0 += a_qk;
  ac1 += a1;
  ac2 += a2;
}

__global__ void __launch_bounds__(kAdjThreads) k_adj_vert(Dims D, double dt, const double *__restrict__ Qh,
                                                  const double *__restrict__ rh, const double *__restrict__ w,
                                                  double *__restrict__ aQ, double *__restrict__ a_rh,
                                                  const double *__restrict__ Qh_pl, const double *__restrict__ rh_pl,
                                                  const double *__restrict__ w_pl, double *__restrict__ aQ_pl,
                                                  double *__restrict__ a_rh_pl, const double *__restrict__ rdgz,
                                                  const double *__restrict__ afact,
                                                  const double *__restrict__ bfact) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = D.lall * D.gall;
  const double *QH, *R, *W;
  double *AQ, *ARH;
  size_t s;
  if (t < ncol) {
    const int l = t / D.gall, c = t % D.gall, G = D.gall_1d;
    if (!inner(D, c % G + 1, c / G + 1)) return;  // halo column: passes through
    const size_t base = (size_t)l * D.kall * D.gall + c;
    QH = Qh + base, R = rh + base, W = w + base, AQ = aQ + base, ARH = a_rh + base, s = D.gall;
  } else if (t < ncol + kLallPl) {
    const size_t base = (size_t)(t - ncol) * D.kall * kGallPl;
    QH = Qh_pl + base, R = rh_pl + base, W = w_pl + base, AQ = aQ_pl + base, ARH = a_rh_pl + base, s = kGallPl;
  } else {
    return;
  }
  const int K = D.kall, kmin = D.kmin, kmax = D.kmax;  // 1-based levels below
  auto X = [&](int k) { return (size_t)(k - 1) * s; };
  const double aTop = AQ[X(K)], aBot = AQ[X(1)];
  extern __shared__ __align__(16) unsigned char adj_raw[];
  AdjRing &ring = *reinterpret_cast<AdjRing *>(adj_raw);
  const int th = threadIdx.x;
  // the levels are taken in the order K, K-1, ..., 1: level j's inputs into slot j % kAdjStages
  auto issue = [&](int j) {
    if (j >= 1) {
      const int sl = j % kAdjStages, kk = (j < kmin) ? kmin : ((j > kmax) ? kmax : j);
      adj_cp8(&ring.v[sl][0][th], QH + X(kk));
      adj_cp8(&ring.v[sl][1][th], R + X(kk));
      adj_cp8(&ring.v[sl][2][th], R + X(j));
      adj_cp8(&ring.v[sl][3][th], W + X(j));
      adj_cp8(&ring.v[sl][4][th], W + X(j < K ? j + 1 : K));
      adj_cp8(&ring.v[sl][5][th], AQ + X(j));
    }
    adj_commit();
  };
#pragma unroll
  for (int d = 0; d < kAdjStages - 1; ++d) issue(K - d);
  auto level = [&](int k) {
    adj_wait<kAdjStages - 2>();  // level k's copies are complete
    const int sl = k % kAdjStages;
    const double vq = ring.v[sl][0][th], vrk = ring.v[sl][1][th], vr = ring.v[sl][2][th];
    const double vw = ring.v[sl][3][th], vw1 = ring.v[sl][4][th], va = ring.v[sl][5][th];
    issue(k - (kAdjStages - 1));  // into the slot of level k + 1, read in the previous call
    VLev v;
    v.qc = vq / vrk;
    v.R = vr;
    v.w = vw;
    v.c1 = v.c2 = v.aO = 0.0;
    if (k >= kmin && k <= kmax) {
      v.c1 = -v.w * dt * rdgz[k - 1] / v.R;
      v.c2 = vw1 * dt * rdgz[k - 1] / v.R;
      double a = va;
      if (k == kmax) a = a + aTop;
      if (k == kmin) a = a + aBot;
      v.aO = a;
    } else if (k == K) {
      v.c1 = -v.w * dt * rdgz[k - 1] / v.R;
    }
    return v;
  };
  // window: levels k+1 (P), k (Z), k-1 (M), k-2 (M2); the Thuburn bounds of a level are
  // recomputed where they are needed instead of carried, which keeps the thread's state small
  VLev P{}, Z = level(K), M = level(K - 1), M2{};
  double aQmZ = 0.0, aQxZ = 0.0, aQmM = 0.0, aQxM = 0.0;  // adjoints of the Qout bounds of k, k-1
  double accP = 0.0, accZ = 0.0, accM = 0.0;             // limiter adjoints into qc(k+1), qc(k), qc(k-1)
  double ac1P = 0.0, ac2P = 0.0;                          // adjoints of ck1, ck2 of level k+1
  double ahP2 = 0.0, ahP = 0.0;                           // post-clamp adjoints of qh(k+2), qh(k+1)
  double aqcTop = 0.0;                                    // adjoint of the ghost qc(kall)
  for (int k = K; k >= kmin; --k) {
    if (k - 2 >= 1) M2 = level(k - 2);
    // qh(k) from the rhogq update of levels k-1 and k
    double ah;
    {
      const bool lo = (k - 1 >= kmin), hi = (k <= kmax);
      const double t1 = lo ? -M.aO * Z.w * dt * rdgz[k - 2] : 0.0;
      const double t2 = hi ? Z.aO * Z.w * dt * rdgz[k - 1] : 0.0;
      ah = (lo && hi) ? t1 + t2 : (lo ? t1 : t2);
    }
    double ac1Z = 0.0, ac2Z = 0.0;
    if (k <= kmax) {
      const VLim LZ = vlim_level(M.qc, Z.qc, P.qc, Z.c1, P.c1, Z.c2);
      // the clamp of qh(k) to the bounds of level k-1 (inflow from below) or k
      if (k >= kmin + 1) {
        const bool below = (LZ.infL != 0.0);
        double Qmx = LZ.Qmx, Qmn = LZ.Qmn;
        if (below) {
          const VLim LM = vlim_level(M2.qc, M.qc, Z.qc, M.c1, Z.c1, M.c2);
          Qmx = LM.Qmx, Qmn = LM.Qmn;
        }
        const double h = afact[k - 1] * Z.qc + bfact[k - 1] * M.qc;
        const double m1 = mn(h, Qmx);
        int sel = (Qmx < h) ? 1 : 0;
        if (Qmn > m1) sel = 2;
        if (sel == 1) {
          if (below) aQxM += ah;
          else aQxZ += ah;
          ah = 0.0;
        } else if (sel == 2) {
          if (below) aQmM += ah;
          else aQmZ += ah;
          ah = 0.0;
        }
      }
      // Qout bounds of level k
      vlim_level_adj(LZ, M.qc, Z.qc, P.qc, aQmZ, aQxZ, accM, accZ, accP, ac1Z, ac2Z);
    }
    // level k+1 is complete
    if (k + 1 == K) {
      aqcTop = accP + afact[K - 1] * ahP;
    } else if (k + 1 <= kmax) {
      double a = accP;
      a += afact[k] * ahP;
      a += bfact[k + 1] * ahP2;
      if (k + 1 == kmax) a += aqcTop;
      const double rR = 1.0 / P.R;
      AQ[X(k + 1)] = P.aO + a * rR;
      double r = ARH[X(k + 1)];
      r += -a * P.qc * rR;
      r += -(ac1P * P.c1 + ac2P * P.c2) * rR;
      ARH[X(k + 1)] = r;
    }
    // shift the window down one level
    P = Z, Z = M, M = M2;
    aQmZ = aQmM, aQxZ = aQxM, aQmM = aQxM = 0.0;
    accP = accZ, accZ = accM, accM = 0.0;
    ac1P = ac1Z, ac2P = ac2Z;
    ahP2 = ahP, ahP = ah;
  }
  // level kmin (now P) with the ghost qc(1) (now Z's accumulator)
  {
    const double aqcBot = accZ + bfact[kmin - 1] * ahP;
    double a = accP;
    a += afact[kmin - 1] * ahP;
    a += bfact[kmin] * ahP2;
    if (kmin == kmax) a += aqcTop;
    a += aqcBot;
    const double rR = 1.0 / P.R;
    AQ[X(kmin)] = P.aO + a * rR;
    double r = ARH[X(kmin)];
    r += -a * P.qc * rR;
    r += -(ac1P * P.c1 + ac2P * P.c2) * rR;
    ARH[X(kmin)] = r;
  }
  AQ[X(1)] = 0.0;
  AQ[X(K)] = 0.0;
  adj_drain();
}

// ---------------------------------------------------------------------------
// Forward recompute of rhogq after the horizontal sub-step, Qh = Q - sum_m flx(m) qa(m),
// with each face's limited value formed from the pre-limit remap value in the
// same operation sequence as the limiter apply (mod_src_tracer.f90:378-410), so
// Qh equals the forward step's value bit for bit without storing the limited faces.
__device__ __forceinline__ double limited_face(const Dims &D, const double *qs, const double *qa0,
                                               const double *qo, const double *cm, size_t off, size_t fs, int oi,
                                               int oj, int a, bool sgp) {
  const int G = D.gall_1d, o = (oj - 1) * G + oi - 1;
  const int nb = (a == 1) ? o + 1 : ((a == 2) ? o + G + 1 : o + G);
  int p[4];
  face_points(D, oi, oj, a, sgp, p);
  const double lo = mn(mn(mn(qs[p[0]], qs[p[1]]), qs[p[2]]), qs[p[3]]);
  const double hi = mx(mx(mx(qs[p[0]], qs[p[1]]), qs[p[2]]), qs[p[3]]);
  const double cc = cm[(size_t)(a - 1) * fs + off + o];
  const double own_min = cc * lo + (1.0 - cc) * kBig, own_max = cc * hi + (1.0 - cc) * (-kBig);
  const double nb_min = cc * kBig + (1.0 - cc) * lo, nb_max = cc * (-kBig) + (1.0 - cc) * hi;
  double v = qa0[(size_t)(a - 1) * fs + off + o];
  v = cc * mn(mx(v, own_min), own_max) + (1.0 - cc) * mn(mx(v, nb_min), nb_max);
  const double on_max = qo[fs + off + nb], on_min = qo[off + nb];
  const double os_max = qo[fs + off + o], os_min = qo[off + o];
  return cc * mx(mn(v, on_max), on_min) + (1.0 - cc) * mx(mn(v, os_max), os_min);
}

__global__ void k_adj_qh(Dims D, const double *__restrict__ q, const double *__restrict__ qa0,
                         const double *__restrict__ qo, const double *__restrict__ cm,
                         const double *__restrict__ flx, const double *__restrict__ Q, double *Qh) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  if (!inner(D, i, j)) return;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  const bool sgp = D.have_sgp[l] != 0;
  const double *qs = q + off;
  // faces 1..3 are owned by (i,j); 4..6 by (i-1,j), (i-1,j-1), (i,j-1) as their faces 1..3
  const int oi[6] = {i, i, i, i - 1, i - 1, i}, oj[6] = {j, j, j, j, j - 1, j - 1};
  double s = flx[off + c] * limited_face(D, qs, qa0, qo, cm, off, fs, oi[0], oj[0], 1, sgp);
  for (int m = 1; m < 6; ++m)
    s = s + flx[(size_t)m * fs + off + c] * limited_face(D, qs, qa0, qo, cm, off, fs, oi[m], oj[m], m % 3 + 1, sgp);
  Qh[off + c] = Q[off + c] - s;
}

// pole centres (mod_src_tracer.f90:412-425 with the Qin bounds kept by the Qout pass)
__global__ void k_adj_qh_pl(int kall, const double *qa0_pl, const double *cm_pl, const double *qo_pl,
                            const double *qin_pl, const double *flx_pl, const double *Qp, double *Qh_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const size_t off = (size_t)t * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  double s = 0.0;
  for (int v = 2; v <= 6; ++v) {
    const double c = cm_pl[off + v - 1];
    double x = qa0_pl[off + v - 1];
    const double i1min = qin_pl[0 * fsp + off + v - 1], i2min = qin_pl[1 * fsp + off + v - 1];
    const double i1max = qin_pl[2 * fsp + off + v - 1], i2max = qin_pl[3 * fsp + off + v - 1];
    x = c * mn(mx(x, i1min), i1max) + (1.0 - c) * mn(mx(x, i2min), i2max);
    x = c * mx(mn(x, qo_pl[fsp + off + v - 1]), qo_pl[off + v - 1]) +
        (1.0 - c) * mx(mn(x, qo_pl[fsp + off]), qo_pl[off]);
    s = (v == 2) ? flx_pl[off + v - 1] * x : s + flx_pl[off + v - 1] * x;
  }
  Qh_pl[off] = Qp[off] - s;
}

// ---------------------------------------------------------------------------
// One face (owner (i,j), a = 1..3): the horizontal update, the limiter apply
// (mod_src_tracer.f90:378-410) and the upwind remap, transposed together.
__global__ void k_adj_face(Dims D, const double *__restrict__ q, const double *__restrict__ qa0,
                           const double *__restrict__ qo, const double *__restrict__ cm,
                           const double *__restrict__ flx, const double *__restrict__ aQ,
                           const double *__restrict__ xc, const double *__restrict__ GRD_x,
                           const double *__restrict__ gr, double *a_flx, double *a_xc, double *a_qo, double *a_q,
                           double *a_gr) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  if (i < D.gmin - 1 || i > D.gmax || j < D.gmin - 1 || j > D.gmax) return;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall, gw = (size_t)D.lall * D.gall;
  const bool sgp = D.have_sgp[l] != 0;
  const double *qs = q + off;
  const bool inC = inner(D, i, j);
  const double aC = inC ? aQ[off + c] : 0.0;
  const int nbs[3] = {c + 1, c + G + 1, c + G};
  const int ni[3] = {i + 1, i + 1, i}, nj[3] = {j, j + 1, j + 1};
  for (int m = 1; m <= 3; ++m) {
    const int nb = nbs[m - 1];
    const bool inN = inner(D, ni[m - 1], nj[m - 1]);
    if (!inC && !inN) continue;
    const double aN = inN ? aQ[off + nb] : 0.0;
    int p[4];
    face_points(D, i, j, m, sgp, p);
    const double qv[4] = {qs[p[0]], qs[p[1]], qs[p[2]], qs[p[3]]};
    const double lo = mn(mn(mn(qv[0], qv[1]), qv[2]), qv[3]);
    const double hi = mx(mx(mx(qv[0], qv[1]), qv[2]), qv[3]);
    const size_t fm = (size_t)(m - 1) * fs + off;
    const double cc = cm[fm + c];
    const double v0 = qa0[fm + c];
    const double v1a = mx(v0, lo);
    int s1 = (lo > v0) ? 1 : 0;
    const double v1 = mn(v1a, hi);
    if (hi < v1a) s1 = 2;
    const int up = (cc != 0.0) ? nb : c;
    const double Qx = qo[fs + off + up], Qn = qo[off + up];
    const double v2a = mn(v1, Qx);
    int s2 = (Qx < v1) ? 1 : 0;
    const double v2 = mx(v2a, Qn);
    if (Qn > v2a) s2 = 2;
    // rhogq -= sum_m flx(m) qa(m) at the owner (face m) and at the neighbour (face m+3)
    const size_t fn = (size_t)(m + 2) * fs + off;
    const double t1 = inC ? -aC * flx[fm + c] : 0.0;
    const double t2 = inN ? -aN * flx[fn + nb] : 0.0;
    const double av = t1 + t2;
    if (inC) a_flx[fm + c] += -aC * v2;
    if (inN) a_flx[fn + nb] += -aN * v2;
    if (av == 0.0) continue;
    if (s2 == 1) {
      atomicAdd(&a_qo[fs + off + up], av);
    } else if (s2 == 2) {
      atomicAdd(&a_qo[off + up], av);
    } else if (s1 == 1) {
      atomicAdd(&a_q[off + p[argmin4(qv)]], av);
    } else if (s1 == 2) {
      atomicAdd(&a_q[off + p[argmax4(qv)]], av);
    } else {  // remap: qa = q(up) + grad(up) . (xc - x(up))
      atomicAdd(&a_q[off + up], av);
      for (int x = 0; x < 3; ++x) {
        const size_t xi = ((size_t)x * 3 + (m - 1)) * fs + off + c;
        atomicAdd(&a_gr[(size_t)x * fs + off + up], av * (xc[xi] - GRD_x[(size_t)x * gw + (size_t)l * D.gall + up]));
        a_xc[xi] += av * gr[(size_t)x * fs + off + up];
      }
    }
  }
}

// pole faces (mod_src_tracer.f90:412-425), one thread per (pole, level, ring face v)
__global__ void k_adj_face_pl(int kall, const double *q_pl, const double *qa0_pl, const double *qo_pl,
                              const double *cm_pl, const double *flx_pl, const double *aQ_pl, const double *xc_pl,
                              const double *GRD_x_pl, const double *gr_pl, double *a_flx_pl, double *a_xc_pl,
                              double *a_qo_pl, double *a_q_pl, double *a_gr_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall * 5) return;
  const int v = t % 5 + 2, kl = t / 5, l = kl / kall;
  const size_t off = (size_t)kl * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  const int vp = (v == 6) ? 2 : v + 1, vm = (v == 2) ? 6 : v - 1;
  const int p[4] = {0, v - 1, vm - 1, vp - 1};
  const double qv[4] = {q_pl[off + p[0]], q_pl[off + p[1]], q_pl[off + p[2]], q_pl[off + p[3]]};
  const double lo = mn(mn(mn(qv[0], qv[1]), qv[2]), qv[3]);
  const double hi = mx(mx(mx(qv[0], qv[1]), qv[2]), qv[3]);
  const double cc = cm_pl[off + v - 1], v0 = qa0_pl[off + v - 1];
  const double v1a = mx(v0, lo);
  int s1 = (lo > v0) ? 1 : 0;
  const double v1 = mn(v1a, hi);
  if (hi < v1a) s1 = 2;
  const int up = (cc != 0.0) ? v - 1 : 0;
  const double Qx = qo_pl[fsp + off + up], Qn = qo_pl[off + up];
  const double v2a = mn(v1, Qx);
  int s2 = (Qx < v1) ? 1 : 0;
  const double v2 = mx(v2a, Qn);
  if (Qn > v2a) s2 = 2;
  const double a = aQ_pl[off];
  const double av = -a * flx_pl[off + v - 1];
  a_flx_pl[off + v - 1] += -a * v2;
  if (av == 0.0) return;
  if (s2 == 1) {
    atomicAdd(&a_qo_pl[fsp + off + up], av);
  } else if (s2 == 2) {
    atomicAdd(&a_qo_pl[off + up], av);
  } else if (s1 == 1) {
    atomicAdd(&a_q_pl[off + p[argmin4(qv)]], av);
  } else if (s1 == 2) {
    atomicAdd(&a_q_pl[off + p[argmax4(qv)]], av);
  } else {
    atomicAdd(&a_q_pl[off + up], av);
    for (int x = 0; x < 3; ++x) {
      const size_t xi = (size_t)x * fsp + off + v - 1;
      atomicAdd(&a_gr_pl[(size_t)x * fsp + off + up],
                av * (xc_pl[xi] - GRD_x_pl[((size_t)x * kLallPl + l) * kGallPl + up]));
      a_xc_pl[xi] += av * gr_pl[(size_t)x * fsp + off + up];
    }
  }
}

// ---------------------------------------------------------------------------
// Qout of one cell (mod_src_tracer.f90:219-301): halo Qout = q, interior the
// Thuburn bounds from the 6 faces' Qin and the Courant numbers.
__global__ void k_adj_qout(Dims D, const double *__restrict__ q, const double *__restrict__ cm,
                           const double *__restrict__ ch, const double *__restrict__ a_qo, double *a_q,
                           double *a_ch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  const double aQn = a_qo[off + c], aQx = a_qo[fs + off + c];
  if (aQn == 0.0 && aQx == 0.0) return;
  if (!inner(D, i, j)) {
    atomicAdd(&a_q[off + c], aQn + aQx);
    return;
  }
  const bool sgp = D.have_sgp[l] != 0;
  const double *qs = q + off;
  const int oi[7] = {0, i, i, i, i - 1, i - 1, i}, oj[7] = {0, j, j, j, j, j - 1, j - 1};
  const int fo[7] = {0, 1, 2, 3, 1, 2, 3};
  double qmn[7], qmx[7], chv[7], chm[7];
  int pmn[7], pmx[7];
  for (int f = 1; f <= 6; ++f) {
    int p[4];
    face_points(D, oi[f], oj[f], fo[f], sgp, p);
    const double qv[4] = {qs[p[0]], qs[p[1]], qs[p[2]], qs[p[3]]};
    const double lo = mn(mn(mn(qv[0], qv[1]), qv[2]), qv[3]);
    const double hi = mx(mx(mx(qv[0], qv[1]), qv[2]), qv[3]);
    const double cmo = cm[(size_t)(fo[f] - 1) * fs + off + p[0]];
    const bool in = (f <= 3) ? (cmo != 0.0) : (cmo == 0.0);
    qmn[f] = in ? lo : kBig;
    qmx[f] = in ? hi : -kBig;
    pmn[f] = in ? p[argmin4(qv)] : -1;
    pmx[f] = in ? p[argmax4(qv)] : -1;
    chv[f] = ch[(size_t)(f - 1) * fs + off + c];
    chm[f] = mn(chv[f], 0.0);
  }
  const double q0 = qs[c];
  double qnmin = q0, qnmax = q0;
  int snmin = 0, snmax = 0;
  for (int f = 1; f <= 6; ++f) {
    if (qmn[f] < qnmin) qnmin = qmn[f], snmin = f;
    if (qmx[f] > qnmax) qnmax = qmx[f], snmax = f;
  }
  const double Cin = chm[1] + chm[2] + chm[3] + chm[4] + chm[5] + chm[6];
  const double Cout = chv[1] - chm[1] + chv[2] - chm[2] + chv[3] - chm[3] + chv[4] - chm[4] + chv[5] - chm[5] +
                      chv[6] - chm[6];
  const double zerosw = 0.5 - sgn(0.5, fabs(Cout) - kEps);
  if (zerosw != 0.0) {
    atomicAdd(&a_q[off + c], aQn + aQx);
    return;
  }
  double CQmin = 0.0, CQmax = 0.0;
  for (int f = 1; f <= 6; ++f) CQmin += chm[f] * qmn[f], CQmax += chm[f] * qmx[f];
  const double S = 1.0 - Cin - Cout;
  const double Nmn = q0 - CQmax - qnmax * S, Nmx = q0 - CQmin - qnmin * S;
  const double Dn = Cout;
  const double aNmn = aQn / Dn, aNmx = aQx / Dn, aD = -(aQn * Nmn + aQx * Nmx) / (Dn * Dn);
  double a_q0 = aNmn + aNmx;
  const double a_qnmax = -aNmn * S, a_qnmin = -aNmx * S;
  const double aS = -aNmn * qnmax - aNmx * qnmin;
  const double aCQmax = -aNmn, aCQmin = -aNmx, aCin = -aS, aCout = -aS + aD;
  if (snmax == 0) a_q0 += a_qnmax;
  else if (pmx[snmax] >= 0) atomicAdd(&a_q[off + pmx[snmax]], a_qnmax);
  if (snmin == 0) a_q0 += a_qnmin;
  else if (pmn[snmin] >= 0) atomicAdd(&a_q[off + pmn[snmin]], a_qnmin);
  atomicAdd(&a_q[off + c], a_q0);
  for (int f = 1; f <= 6; ++f) {
    double achm = aCin;
    if (pmn[f] >= 0) atomicAdd(&a_q[off + pmn[f]], aCQmin * chm[f]), achm += aCQmin * qmn[f];
    if (pmx[f] >= 0) atomicAdd(&a_q[off + pmx[f]], aCQmax * chm[f]), achm += aCQmax * qmx[f];
    const double dchm = (0.0 < chv[f]) ? 0.0 : 1.0;
    a_ch[(size_t)(f - 1) * fs + off + c] += aCout * (1.0 - dchm) + achm * dchm;
  }
}

// pole centre Qout (mod_src_tracer.f90:307-367), one thread per (pole, level)
__global__ void k_adj_qout_pl(int kall, const double *q_pl, const double *cm_pl, const double *ch_pl,
                              const double *a_qo_pl, double *a_q_pl, double *a_ch_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const size_t off = (size_t)t * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  const double aQn = a_qo_pl[off], aQx = a_qo_pl[fsp + off];
  if (aQn == 0.0 && aQx == 0.0) return;
  const double *qs = q_pl + off;
  double qmn[7], qmx[7];
  int pmn[7], pmx[7];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1, vm = (v == 2) ? 6 : v - 1;
    const int p[4] = {0, v - 1, vm - 1, vp - 1};
    const double qv[4] = {qs[p[0]], qs[p[1]], qs[p[2]], qs[p[3]]};
    const double lo = mn(mn(mn(qv[0], qv[1]), qv[2]), qv[3]);
    const double hi = mx(mx(mx(qv[0], qv[1]), qv[2]), qv[3]);
    const bool in = cm_pl[off + v - 1] != 0.0;
    qmn[v] = in ? lo : kBig;
    qmx[v] = in ? hi : -kBig;
    pmn[v] = in ? p[argmin4(qv)] : -1;
    pmx[v] = in ? p[argmax4(qv)] : -1;
  }
  const double q0 = qs[0];
  double qnmin = q0, qnmax = q0;
  int snmin = 0, snmax = 0;
  for (int v = 2; v <= 6; ++v) {
    if (qmn[v] < qnmin) qnmin = qmn[v], snmin = v;
    if (qmx[v] > qnmax) qnmax = qmx[v], snmax = v;
  }
  double Cin = 0.0, Cout = 0.0, CQmax = 0.0, CQmin = 0.0, chmk[7];
  for (int v = 2; v <= 6; ++v) {
    chmk[v] = cm_pl[off + v - 1] * ch_pl[off + v - 1];
    Cin = Cin + chmk[v];
    Cout = Cout - chmk[v] + ch_pl[off + v - 1];
    CQmin = CQmin + chmk[v] * qmn[v];
    CQmax = CQmax + chmk[v] * qmx[v];
  }
  const double zerosw = 0.5 - sgn(0.5, fabs(Cout) - kEps);
  if (zerosw != 0.0) {
    a_q_pl[off] += aQn + aQx;
    return;
  }
  const double S = 1.0 - Cin - Cout, Dn = Cout;
  const double Nmn = q0 - CQmax - qnmax * S, Nmx = q0 - CQmin - qnmin * S;
  const double aNmn = aQn / Dn, aNmx = aQx / Dn, aD = -(aQn * Nmn + aQx * Nmx) / (Dn * Dn);
  double a_q0 = aNmn + aNmx;
  const double a_qnmax = -aNmn * S, a_qnmin = -aNmx * S;
  const double aS = -aNmn * qnmax - aNmx * qnmin;
  const double aCQmax = -aNmn, aCQmin = -aNmx, aCin = -aS, aCout = -aS + aD;
  if (snmax == 0) a_q0 += a_qnmax;
  else if (pmx[snmax] >= 0) a_q_pl[off + pmx[snmax]] += a_qnmax;
  if (snmin == 0) a_q0 += a_qnmin;
  else if (pmn[snmin] >= 0) a_q_pl[off + pmn[snmin]] += a_qnmin;
  a_q_pl[off] += a_q0;
  for (int v = 2; v <= 6; ++v) {
    const double cc = cm_pl[off + v - 1];
    double achm = aCin - aCout;
    if (pmn[v] >= 0) a_q_pl[off + pmn[v]] += aCQmin * chmk[v], achm += aCQmin * qmn[v];
    if (pmx[v] >= 0) a_q_pl[off + pmx[v]] += aCQmax * chmk[v], achm += aCQmax * qmx[v];
    a_ch_pl[off + v - 1] += aCout + achm * cc;
  }
}

// ---------------------------------------------------------------------------
// gradient stencil (mod_oprt.f90:499-734 coefficients), transposed as a gather:
// point p collects coef(c, n) a_grad(c) from the interior cells c whose n-th
// stencil point it is.
__global__ void k_adj_grad(Dims D, const double *__restrict__ cg, const double *__restrict__ a_gr, double *a_q) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  const int d[7] = {0, 1, G + 1, G, -1, -G - 1, -G};
  double s = 0.0;
  bool any = false;
  for (int n = 0; n < 7; ++n) {
    const int c = p - d[n];
    if (c < 0 || c >= D.gall || !inner(D, c % G + 1, c / G + 1)) continue;
    for (int x = 0; x < 3; ++x) {
      const double a = a_gr[(size_t)x * fs + off + c];
      if (a == 0.0) continue;
      s += cg[(((size_t)l * 3 + x) * 7 + n) * D.gall + c] * a;
      any = true;
    }
  }
  if (any) a_q[off + p] += s;
}
__global__ void k_adj_grad_pl(int kall, const double *cg_pl, const double *a_gr_pl, double *a_q_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const int l = t / kall;
  const size_t off = (size_t)t * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  for (int x = 0; x < 3; ++x) {
    const double a = a_gr_pl[(size_t)x * fsp + off];
    const double *cx = cg_pl + ((size_t)l * 3 + x) * 6;
    a_q_pl[off] += cx[0] * a;
    for (int v = 2; v <= 6; ++v) a_q_pl[off + v - 1] += cx[v - 1] * a;
  }
}

// q = Q / rho: a_Q += a_q / rho, a_rho -= a_q q / rho (regions and poles in one launch)
__global__ void k_adj_div(long long n3, int n3p, const double *a_q, const double *q, const double *rho,
                          const double *a_q_pl, const double *q_pl, const double *rho_pl, double *aQ, double *aQp,
                          double *a_rho, double *a_rho_pl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n3) {
    const double a = a_q[t];
    if (a == 0.0) return;
    aQ[t] += a / rho[t];
    a_rho[t] += -a * q[t] / rho[t];
  } else if (t < n3 + n3p) {
    const long long u = t - n3;
    const double a = a_q_pl[u];
    if (a == 0.0) return;
    aQp[u] += a / rho_pl[u];
    a_rho_pl[u] += -a * q_pl[u] / rho_pl[u];
  }
}

// rho_h = rho - sum_m flx(m) and ch(m) = flx(m) / rho: adjoints to flx and rho
__global__ void k_adj_rhoh_ch(Dims D, const double *rho, const double *ch, const double *a_rh, const double *a_ch,
                              double *a_flx, double *a_rho) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, G = D.gall_1d;
  const size_t off = (size_t)kl * D.gall + c, fs = (size_t)D.lall * D.kall * D.gall;
  const double ah = a_rh[off];
  double ar = a_rho[off] + ah;
  const bool in = inner(D, c % G + 1, c / G + 1);
  const double r = rho[off];
  for (int m = 0; m < 6; ++m) {
    double f = a_flx[m * fs + off];
    if (in) f += -ah;
    const double a = a_ch[m * fs + off];
    if (a != 0.0) {
      f += a / r;
      ar += -a * ch[m * fs + off] / r;
    }
    a_flx[m * fs + off] = f;
  }
  a_rho[off] = ar;
}
__global__ void k_adj_rhoh_ch_pl(int kall, const double *rho_pl, const double *ch_pl, const double *a_rh_pl,
                                 const double *a_ch_pl, double *a_flx_pl, double *a_rho_pl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const size_t off = (size_t)t * kGallPl;
  const double ah = a_rh_pl[off];
  a_rho_pl[off] += ah;
  for (int v = 2; v <= 6; ++v) a_flx_pl[off + v - 1] += -ah;
  const double r = rho_pl[off];
  for (int v = 2; v <= 6; ++v) {
    const double a = a_ch_pl[off + v - 1];
    if (a == 0.0) continue;
    a_flx_pl[off + v - 1] += a / r;
    a_rho_pl[off] += -a * ch_pl[off + v - 1] / r;
  }
}

// ---------------------------------------------------------------------------
// horizontal_flux.  Triangle values (:141-201): TI(ij) from (ij, ip1j, ip1jp1),
// TJ(ij) from (ij, ip1jp1, ijp1), TI(gmin-1,gmin-1) = TJ(gmin,gmin-1) on a
// singular region.  A face sums its two triangles: AI(ij) = TJ(ijm1) + TI(ij),
// AIJ(ij) = TI(ij) + TJ(ij), AJ(ij) = TJ(ij) + TI(im1j).
struct Fld {
  const double *f[4];  // rho, rhovx, rhovy, rhovz
};
struct Tv {
  double v[4];
};

__device__ __forceinline__ Tv tri(const Dims &D, const Fld &F, const double *GT, int l, size_t off, int c, int t) {
  // t = 1 (TI), 2 (TJ); c 0-based owner
  const size_t gw = (size_t)D.gall * D.lall;
  const int G = D.gall_1d;
  const double w1 = GT[((size_t)(W1 - 1) * 2 + (t - 1)) * gw + (size_t)l * D.gall + c];
  const double w2 = GT[((size_t)(W2 - 1) * 2 + (t - 1)) * gw + (size_t)l * D.gall + c];
  const double w3 = GT[((size_t)(W3 - 1) * 2 + (t - 1)) * gw + (size_t)l * D.gall + c];
  const int b = (t == 1) ? c + 1 : c + G + 1, e = (t == 1) ? c + G + 1 : c + G;
  Tv r;
  for (int x = 0; x < 4; ++x) r.v[x] = F.f[x][off + c] * w1 + F.f[x][off + b] * w2 + F.f[x][off + e] * w3;
  return r;
}
__device__ __forceinline__ Tv triI(const Dims &D, const Fld &F, const double *GT, int l, size_t off, int c, bool sgp) {
  const int G = D.gall_1d;
  if (sgp && c == (D.gmin - 2) * G + (D.gmin - 2)) return tri(D, F, GT, l, off, c + 1, 2);
  return tri(D, F, GT, l, off, c, 1);
}

// adjoint of one face's (flux, xc) -> its two triangles (aT gets += for both)
__device__ __forceinline__ void face_adj(const Dims &D, const Geo<double> &g, const double *a_flx,
                                         const double *a_xc, double dt, int l, size_t off, size_t fs, int o, int a,
                                         bool sgp, const Tv &p, const Tv &q, Tv &ap) {
  const size_t gw = (size_t)D.gall * D.lall;
  const int G = D.gall_1d;
  const int nb = (a == 1) ? o + 1 : ((a == 2) ? o + G + 1 : o + G);
  const double rsum = p.v[0] + q.v[0];
  double vs[3];
  for (int x = 0; x < 3; ++x) vs[x] = p.v[x + 1] + q.v[x + 1];
  const double rr = 1.0 / mx(rsum, kEps);
  double aflux = a_flx[(size_t)(a - 1) * fs + off + o] * g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + o] * dt;
  const bool sg0 = sgp && a == 3 && nb == (D.gmin - 1) * G + (D.gmin - 1);
  if (!sg0)
    aflux += -a_flx[(size_t)(a + 2) * fs + off + nb] * g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + nb] *
             dt;
  double avs[3], arr = 0.0;
  for (int x = 0; x < 3; ++x)
    avs[x] = 0.5 * aflux * g.GMTR_a[((size_t)x * 3 + (a - 1)) * gw + (size_t)l * D.gall + o];
  for (int x = 0; x < 3; ++x) {
    const double ax = a_xc[((size_t)x * 3 + (a - 1)) * fs + off + o];
    avs[x] += -ax * rr * dt * 0.5;
    arr += -ax * vs[x] * dt * 0.5;
  }
  const double ars = (rsum > kEps) ? -arr * rr * rr : 0.0;
  ap.v[0] += ars;
  for (int x = 0; x < 3; ++x) ap.v[x + 1] += avs[x];
}

// triangle adjoints of owner p: TI(p) from AI(p), AIJ(p), AJ(p+1); TJ(p) from AI(p+G), AIJ(p), AJ(p)
__global__ void k_adj_tri(Dims D, Geo<double> g, Fld F, const double *a_flx, const double *a_xc, double dt,
                          double *aT) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const int i = c % G + 1, j = c / G + 1;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall;
  Tv aI{}, aJ{};
  const int lo = D.gmin - 1, hi = D.gmax;
  if (i >= lo && i <= hi && j >= lo && j <= hi) {
    const bool sgp = D.have_sgp[l] != 0;
    const double *GT = g.GMTR_t;
    const Tv tI = triI(D, F, GT, l, off, c, sgp), tJ = tri(D, F, GT, l, off, c, 2);
    if (j >= D.gmin) face_adj(D, g, a_flx, a_xc, dt, l, off, fs, c, 1, sgp, tri(D, F, GT, l, off, c - G, 2), tI, aI);
    {
      Tv a2{};
      face_adj(D, g, a_flx, a_xc, dt, l, off, fs, c, 2, sgp, tI, tJ, a2);
      for (int x = 0; x < 4; ++x) aI.v[x] += a2.v[x], aJ.v[x] += a2.v[x];
    }
    if (i + 1 >= D.gmin && i + 1 <= hi)
      face_adj(D, g, a_flx, a_xc, dt, l, off, fs, c + 1, 3, sgp, tri(D, F, GT, l, off, c + 1, 2), tI, aI);
    if (j + 1 >= D.gmin && j + 1 <= hi)
      face_adj(D, g, a_flx, a_xc, dt, l, off, fs, c + G, 1, sgp, tJ, triI(D, F, GT, l, off, c + G, sgp), aJ);
    if (i >= D.gmin) face_adj(D, g, a_flx, a_xc, dt, l, off, fs, c, 3, sgp, tJ, triI(D, F, GT, l, off, c - 1, sgp), aJ);
  }
  for (int x = 0; x < 4; ++x) {
    aT[(size_t)x * fs + off + c] = aI.v[x];
    aT[(size_t)(4 + x) * fs + off + c] = aJ.v[x];
  }
}

// fields from the triangles: point p is ij of TI/TJ(p) (W1), ip1j of TI(p-1) (W2),
// ip1jp1 of TI(p-G-1) (W3) and TJ(p-G-1) (W2), ijp1 of TJ(p-G) (W3); on a singular
// region TI(gmin-1,gmin-1) is TJ(gmin,gmin-1)
__global__ void k_adj_fields(Dims D, const double *GT, const double *aT, double *a0, double *a1, double *a2,
                             double *a3) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall, G = D.gall_1d;
  const size_t off = (size_t)kl * D.gall, fs = (size_t)D.lall * D.kall * D.gall, gw = (size_t)D.gall * D.lall;
  const bool sgp = D.have_sgp[l] != 0;
  const int sg = (D.gmin - 2) * G + (D.gmin - 2);
  auto ok = [&](int c) {
    if (c < 0 || c >= D.gall) return false;
    const int i = c % G + 1, j = c / G + 1;
    return i >= D.gmin - 1 && i <= D.gmax && j >= D.gmin - 1 && j <= D.gmax;
  };
  auto w = [&](int c, int t, int wi) { return GT[((size_t)(wi - 1) * 2 + (t - 1)) * gw + (size_t)l * D.gall + c]; };
  auto aI = [&](int c, int x) { return (sgp && c == sg) ? 0.0 : aT[(size_t)x * fs + off + c]; };
  auto aJ = [&](int c, int x) {
    double v = aT[(size_t)(4 + x) * fs + off + c];
    if (sgp && c == sg + 1) v += aT[(size_t)x * fs + off + sg];
    return v;
  };
  double *out[4] = {a0, a1, a2, a3};
  for (int x = 0; x < 4; ++x) {
    double s = 0.0;
    if (ok(p)) s += aI(p, x) * w(p, TI, W1) + aJ(p, x) * w(p, TJ, W1);
    if (ok(p - 1)) s += aI(p - 1, x) * w(p - 1, TI, W2);
    if (ok(p - G - 1)) s += aI(p - G - 1, x) * w(p - G - 1, TI, W3) + aJ(p - G - 1, x) * w(p - G - 1, TJ, W2);
    if (ok(p - G)) s += aJ(p - G, x) * w(p - G, TJ, W3);
    out[x][off + p] += s;
  }
}

// pole faces of horizontal_flux (:326-374), one thread per (pole, level)
__global__ void k_adj_flux_pl(int kall, Geo<double> g, Fld F, const double *a_flx_pl, const double *a_xc_pl,
                              double dt, double *a0, double *a1, double *a2, double *a3) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * kall) return;
  const int l = t / kall;
  const size_t off = (size_t)t * kGallPl, fsp = (size_t)kLallPl * kall * kGallPl;
  auto GT = [&](int v, int wi) { return g.GMTR_t_pl[((size_t)(wi - 1) * kLallPl + l) * kGallPl + (v - 1)]; };
  auto GA = [&](int v, int h) { return g.GMTR_a_pl[((size_t)(h - 1) * kLallPl + l) * kGallPl + (v - 1)]; };
  const double rarea = g.GMTR_p_pl[((size_t)(P_RAREA - 1) * kLallPl + l) * kGallPl + 0];
  double tt[7][4], at[7][4];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    for (int x = 0; x < 4; ++x) {
      tt[v][x] = F.f[x][off] * GT(v, W1) + F.f[x][off + v - 1] * GT(v, W2) + F.f[x][off + vp - 1] * GT(v, W3);
      at[v][x] = 0.0;
    }
  }
  for (int v = 2; v <= 6; ++v) {
    const int vm = (v == 2) ? 6 : v - 1;
    const double rsum = tt[vm][0] + tt[v][0];
    const double rr = 1.0 / mx(rsum, kEps);
    const double aflux = a_flx_pl[off + v - 1] * rarea * dt;
    double avs[3], arr = 0.0;
    for (int x = 0; x < 3; ++x) avs[x] = 0.5 * aflux * GA(v, HNX + x);
    for (int x = 0; x < 3; ++x) {
      const double vsx = tt[vm][x + 1] + tt[v][x + 1];
      const double ax = a_xc_pl[(size_t)x * fsp + off + v - 1];
      avs[x] += -ax * rr * dt * 0.5;
      arr += -ax * vsx * dt * 0.5;
    }
    const double ars = (rsum > kEps) ? -arr * rr * rr : 0.0;
    at[vm][0] += ars, at[v][0] += ars;
    for (int x = 0; x < 3; ++x) at[vm][x + 1] += avs[x], at[v][x + 1] += avs[x];
  }
  double *out[4] = {a0, a1, a2, a3};
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    for (int x = 0; x < 4; ++x) {
      out[x][off] += at[v][x] * GT(v, W1);
      out[x][off + v - 1] += at[v][x] * GT(v, W2);
      out[x][off + vp - 1] += at[v][x] * GT(v, W3);
    }
  }
}

dim3 slab(const Dims &D, int th) { return dim3((D.gall + th - 1) / th, D.kall * D.lall); }

void fill_adj(const StepCtx &S, double *a, double *a_pl, int vmax, cudaStream_t st) {
  const Dims &D = S.D;
  const long long total = (long long)S.plan.n * D.kall * vmax;
  if (total == 0) return;
  k_fill_adj<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(S.plan.n, S.plan.dst, S.plan.src, D.gall * D.lall,
                                                              D.gall, D.lall, D.kall, vmax, a, a_pl);
}

}  // namespace

int step_adjoint(StepCtx &S, const AdjScratch &A, int ntr, double dt, const double *rhog, const double *rhog_pl,
                 const double *rhogq, const double *rhogq_pl, const double *vx, const double *vx_pl,
                 const double *vy, const double *vy_pl, const double *vz, const double *vz_pl, const double *w,
                 const double *w_pl, double *a_rhog, double *a_rhog_pl, double *a_rhogq, double *a_rhogq_pl,
                 double *a_vx, double *a_vx_pl, double *a_vy, double *a_vy_pl, double *a_vz, double *a_vz_pl,
                 cudaStream_t st, long long &launches) {
  const Dims &D = S.D;
  if (D.kall < 4 || D.kmax <= D.kmin) return ICA_ERR_ARG;
  const size_t n3 = (size_t)D.gall * D.kall * D.lall, n3p = (size_t)kGallPl * D.kall * kLallPl;
  const size_t B = sizeof(double);
  const int T = 128;
  const unsigned nbl = (unsigned)((kLallPl * D.kall + 127) / 128);
  // ---- forward recompute of the step-level intermediates
  FluxIn<double> fin{rhog, rhog_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl};
  FluxOut<double> fout{S.flx, S.flx_pl, S.xc, S.xc_pl};
  launch_horizontal_flux<double>(D, fin, fout, S.geo, dt, st);
  launch_courant(S, rhog, rhog_pl, st);
  cudaMemcpyAsync(A.rh, rhog, n3 * B, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(A.rh_pl, rhog_pl, n3p * B, cudaMemcpyDeviceToDevice, st);
  launch_update_rho(S, A.rh, A.rh_pl, st);
  cudaMemsetAsync(A.a_flx, 0, 6 * n3 * B, st);
  cudaMemsetAsync(A.a_flx_pl, 0, n3p * B, st);
  cudaMemsetAsync(A.a_xc, 0, 9 * n3 * B, st);
  cudaMemsetAsync(A.a_xc_pl, 0, 3 * n3p * B, st);
  cudaMemsetAsync(A.a_ch, 0, 6 * n3 * B, st);
  cudaMemsetAsync(A.a_ch_pl, 0, n3p * B, st);
  launches += 6;
  // ---- the final halo fill and the density part of the vertical sub-step
  fill_adj(S, a_rhog, a_rhog_pl, 1, st);
  fill_adj(S, a_rhogq, a_rhogq_pl, ntr, st);
  const int npt = D.lall * D.gall + kLallPl * kGallPl;
  k_adj_vrho<<<(npt + 127) / 128, 128, 0, st>>>(D, a_rhog, a_rhog_pl, A.a_rh, A.a_rh_pl);
  launches += 3;
  // ---- tracer by tracer: recompute the horizontal sub-step, then transpose it
  LimIn<double> lin{S.q, S.q_pl, S.zero, S.zero_pl, S.ch, S.ch_pl, S.cm, S.cm_pl};
  const int ncol = D.lall * D.gall + kLallPl;
  for (int t = 0; t < ntr; ++t) {
    const double *Q = rhogq + t * n3, *Qp = rhogq_pl + t * n3p;
    double *aQ = a_rhogq + t * n3, *aQp = a_rhogq_pl + t * n3p;
    launch_divide(S, Q, Qp, rhog, rhog_pl, st);
    launch_gradient(S, st);
    launch_remap(S, st);
    launch_hlim_qout<double>(D, lin, S.qout, S.qout_pl, S.qin_pl, st);
    launch_gather<double>(D, S.plan.n, S.plan.dst, S.plan.src, D.kall, 2, S.qout, S.qout_pl, st);
    k_adj_qh<<<slab(D, T), T, 0, st>>>(D, S.q, S.qa, S.qout, S.cm, S.flx, Q, A.Qh);
    k_adj_qh_pl<<<nbl, 128, 0, st>>>(D.kall, S.qa_pl, S.cm_pl, S.qout_pl, S.qin_pl, S.flx_pl, Qp, A.Qh_pl);
    // vertical sub-step: aQ becomes the adjoint of rhogq after the horizontal sub-step
    k_adj_vert<<<(ncol + kAdjThreads - 1) / kAdjThreads, kAdjThreads, (int)sizeof(AdjRing), st>>>(D, dt, A.Qh, A.rh, w, aQ, A.a_rh, A.Qh_pl, A.rh_pl, w_pl, aQp,
                                                   A.a_rh_pl, S.rdgz, S.afact, S.bfact);
    cudaMemsetAsync(A.a_q, 0, n3 * B, st);
    cudaMemsetAsync(A.a_q_pl, 0, n3p * B, st);
    cudaMemsetAsync(A.a_gr, 0, 3 * n3 * B, st);
    cudaMemsetAsync(A.a_gr_pl, 0, 3 * n3p * B, st);
    cudaMemsetAsync(A.a_qo, 0, 2 * n3 * B, st);
    cudaMemsetAsync(A.a_qo_pl, 0, 2 * n3p * B, st);
    k_adj_face<<<slab(D, T), T, 0, st>>>(D, S.q, S.qa, S.qout, S.cm, S.flx, aQ, S.xc, S.GRD_x, S.grad, A.a_flx,
                                         A.a_xc, A.a_qo, A.a_q, A.a_gr);
    k_adj_face_pl<<<(unsigned)((kLallPl * D.kall * 5 + 127) / 128), 128, 0, st>>>(
        D.kall, S.q_pl, S.qa_pl, S.qout_pl, S.cm_pl, S.flx_pl, aQp, S.xc_pl, S.GRD_x_pl, S.grad_pl, A.a_flx_pl,
        A.a_xc_pl, A.a_qo_pl, A.a_q_pl, A.a_gr_pl);
    fill_adj(S, A.a_qo, A.a_qo_pl, 2, st);
    k_adj_qout<<<slab(D, T), T, 0, st>>>(D, S.q, S.cm, S.ch, A.a_qo, A.a_q, A.a_ch);
    k_adj_qout_pl<<<nbl, 128, 0, st>>>(D.kall, S.q_pl, S.cm_pl, S.ch_pl, A.a_qo_pl, A.a_q_pl, A.a_ch_pl);
    fill_adj(S, A.a_gr, A.a_gr_pl, 3, st);
    k_adj_grad<<<slab(D, T), T, 0, st>>>(D, S.cg, A.a_gr, A.a_q);
    k_adj_grad_pl<<<nbl, 128, 0, st>>>(D.kall, S.cg_pl, A.a_gr_pl, A.a_q_pl);
    k_adj_div<<<(unsigned)((n3 + n3p + 255) / 256), 256, 0, st>>>((long long)n3, (int)n3p, A.a_q, S.q, rhog,
                                                                  A.a_q_pl, S.q_pl, rhog_pl, aQ, aQp, a_rhog,
                                                                  a_rhog_pl);
    launches += 27;
  }
  // ---- density update and Courant numbers, then horizontal_flux
  k_adj_rhoh_ch<<<slab(D, T), T, 0, st>>>(D, rhog, S.ch, A.a_rh, A.a_ch, A.a_flx, a_rhog);
  k_adj_rhoh_ch_pl<<<nbl, 128, 0, st>>>(D.kall, rhog_pl, S.ch_pl, A.a_rh_pl, A.a_ch_pl, A.a_flx_pl, a_rhog_pl);
  const Fld F{{rhog, vx, vy, vz}};
  const Fld Fp{{rhog_pl, vx_pl, vy_pl, vz_pl}};
  k_adj_tri<<<slab(D, T), T, 0, st>>>(D, S.geo, F, A.a_flx, A.a_xc, dt, A.aT);
  k_adj_fields<<<slab(D, T), T, 0, st>>>(D, S.geo.GMTR_t, A.aT, a_rhog, a_vx, a_vy, a_vz);
  k_adj_flux_pl<<<nbl, 128, 0, st>>>(D.kall, S.geo, Fp, A.a_flx_pl, A.a_xc_pl, dt, a_rhog_pl, a_vx_pl, a_vy_pl,
                                     a_vz_pl);
  launches += 5;
  return ICA_OK;
}

}  // namespace icoadv
