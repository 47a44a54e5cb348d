// Plain kernels: one CUDA kernel per reference subroutine, FP64 (RP = DP) and
// FP32 (RP = SP), same argument meaning and array layout as the reference.
//
//   horizontal_flux            dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-379
//   horizontal_limiter_thuburn dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-430
//   vertical_limiter_thuburn   dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-243
//   COMM_data_transfer         communication/src/mod_comm.f90:1506-1891 (as a gather)
//
// This file is compiled with --fmad=false: every expression keeps the
// reference's operation order and no multiply-add is contracted, so the FP64
// results equal a non-contracting CPU build of the reference bit for bit.
//
// Thread mapping.  The reference loops over faces and scatters each face
// value to both cells (flx_h(ij,1) and flx_h(ip1j,4), Qin(ij,1) and
// Qin(ip1j,4), q_a(ij,1) and q_a(ip1j,4)).  Here one thread owns one cell
// (i,j) of one (k,l) slab, evaluates the three faces the reference attaches to
// that cell, and writes both sides; every output element has exactly one
// writer, and halo elements that no face loop reaches get the zero the
// reference writes first.  Index (i,j) is 1-based as in the reference,
// ij = (j-1)*gall_1d + i, arrays are addressed with ij-1.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "plain_kernels.cuh"

namespace icoadv {

template <typename T> struct Num;
template <> struct Num<double> {
  static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
  static __device__ __forceinline__ double big() { return DBL_MAX; }
};
template <> struct Num<float> {
  static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
  static __device__ __forceinline__ float big() { return FLT_MAX; }
};

// Fortran MIN/MAX of two values and SIGN(a,b) with IEEE signed zero.
template <typename T> __device__ __forceinline__ T mn(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T mx(T a, T b) { return (b > a) ? b : a; }
template <typename T> __device__ __forceinline__ T fsign(T a, T b) { return copysign(fabs(a), b); }

// ---------------------------------------------------------------------------
// horizontal_flux
struct TriVal {
  double r, x, y, z;
};
template <typename T> struct Tri {
  T r, x, y, z;
};

template <typename T>
__device__ __forceinline__ Tri<T> tri_TI(const Dims &D, const FluxIn<T> &in, const Geo<T> &g, int l,
                                         size_t off, int ij) {
  // rhot_TI(ij) = rho(ij)*W1 + rho(ip1j)*W2, then + rho(ip1jp1)*W3   (:146-153, :171-174)
  const size_t gw = (size_t)D.gall * D.lall;
  const T w1 = g.GMTR_t[(size_t)(W1 - 1) * 2 * gw + (size_t)(TI - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const T w2 = g.GMTR_t[(size_t)(W2 - 1) * 2 * gw + (size_t)(TI - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const T w3 = g.GMTR_t[(size_t)(W3 - 1) * 2 * gw + (size_t)(TI - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const int a = ij - 1, b = ij, c = ij + D.gall_1d;
  Tri<T> t;
  t.r = in.rho[off + a] * w1 + in.rho[off + b] * w2;
  t.x = in.rhovx[off + a] * w1 + in.rhovx[off + b] * w2;
  t.y = in.rhovy[off + a] * w1 + in.rhovy[off + b] * w2;
  t.z = in.rhovz[off + a] * w1 + in.rhovz[off + b] * w2;
  t.r = t.r + in.rho[off + c] * w3;
  t.x = t.x + in.rhovx[off + c] * w3;
  t.y = t.y + in.rhovy[off + c] * w3;
  t.z = t.z + in.rhovz[off + c] * w3;
  return t;
}

template <typename T>
__device__ __forceinline__ Tri<T> tri_TJ(const Dims &D, const FluxIn<T> &in, const Geo<T> &g, int l,
                                         size_t off, int ij) {
  // rhot_TJ(ij) = rho(ij)*W1, then + rho(ip1jp1)*W2 + rho(ijp1)*W3   (:155-158, :176-183)
  const size_t gw = (size_t)D.gall * D.lall;
  const T w1 = g.GMTR_t[(size_t)(W1 - 1) * 2 * gw + (size_t)(TJ - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const T w2 = g.GMTR_t[(size_t)(W2 - 1) * 2 * gw + (size_t)(TJ - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const T w3 = g.GMTR_t[(size_t)(W3 - 1) * 2 * gw + (size_t)(TJ - 1) * gw + (size_t)l * D.gall + (ij - 1)];
  const int a = ij - 1, c = ij + D.gall_1d, e = ij + D.gall_1d - 1;
  Tri<T> t;
  t.r = in.rho[off + a] * w1;
  t.x = in.rhovx[off + a] * w1;
  t.y = in.rhovy[off + a] * w1;
  t.z = in.rhovz[off + a] * w1;
  t.r = t.r + in.rho[off + c] * w2 + in.rho[off + e] * w3;
  t.x = t.x + in.rhovx[off + c] * w2 + in.rhovx[off + e] * w3;
  t.y = t.y + in.rhovy[off + c] * w2 + in.rhovy[off + e] * w3;
  t.z = t.z + in.rhovz[off + c] * w2 + in.rhovz[off + e] * w3;
  return t;
}

// TI with the singular-point override rhot_TI(gmin-1,gmin-1) = rhot_TJ(gmin,gmin-1)   (:188-201)
template <typename T>
__device__ __forceinline__ Tri<T> tri_TI_s(const Dims &D, const FluxIn<T> &in, const Geo<T> &g, int l,
                                           size_t off, int i, int j, bool sgp) {
  const int ij = (j - 1) * D.gall_1d + i;
  if (sgp && i == D.gmin - 1 && j == D.gmin - 1) return tri_TJ(D, in, g, l, off, ij + 1);
  return tri_TI(D, in, g, l, off, ij);
}

template <typename T>
__global__ void k_horizontal_flux(Dims D, FluxIn<T> in, FluxOut<T> out, Geo<T> g, T dt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y;  // l*kall + k
  const int l = kl / D.kall;
  const int i = c % D.gall_1d + 1, j = c / D.gall_1d + 1;
  const int ij = c + 1, G = D.gall_1d, gmin = D.gmin, gmax = D.gmax;
  const size_t off = (size_t)kl * D.gall;                  // (k,l) slab of a 3-D field
  const size_t fs = (size_t)D.lall * D.kall * D.gall;      // stride of the last dimension
  const size_t gw = (size_t)D.gall * D.lall;               // geometry stride
  const bool sgp = D.have_sgp[l] != 0;
  const T EPS = Num<T>::eps();
  const T rarea_ij = g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + c];
  auto HN = [&](int cell, int a, int h) -> T {
    return g.GMTR_a[((size_t)(h - 1) * 3 + (a - 1)) * gw + (size_t)l * D.gall + (cell - 1)];
  };
  auto XR = [&](int cell, int a, int x) -> T {
    return g.GRD_xr[((size_t)(x - 1) * 3 + (a - 1)) * gw + (size_t)l * D.gall + (cell - 1)];
  };
  auto store_xc = [&](int a, T x, T y, T z) {
    out.GRD_xc[((size_t)0 * 3 + (a - 1)) * fs + off + c] = x;
    out.GRD_xc[((size_t)1 * 3 + (a - 1)) * fs + off + c] = y;
    out.GRD_xc[((size_t)2 * 3 + (a - 1)) * fs + off + c] = z;
  };
  auto face = [&](const Tri<T> &p, const Tri<T> &q, int a, T &rrhoa2, T &vx, T &vy, T &vz) -> T {
    rrhoa2 = T(1) / mx(p.r + q.r, EPS);
    vx = p.x + q.x;
    vy = p.y + q.y;
    vz = p.z + q.z;
    return T(0.5) * (vx * HN(ij, a, HNX) + vy * HN(ij, a, HNY) + vz * HN(ij, a, HNZ));
  };
  const bool inI = (i >= gmin && i <= gmax), inJ = (j >= gmin && j <= gmax);
  const bool extI = (i >= gmin - 1 && i <= gmax), extJ = (j >= gmin - 1 && j <= gmax);
  // AI face of (i,j): flx_h(ij,1), flx_h(ip1j,4), GRD_xc(ij,AI)   (:235-257)
  if (inJ && extI) {
    T r2, vx, vy, vz;
    const Tri<T> tj = tri_TJ(D, in, g, l, off, ij - G);  // TJ(ijm1): j-1 >= gmin-1, never singular
    const Tri<T> ti = tri_TI_s(D, in, g, l, off, i, j, sgp);
    const T flux = face(tj, ti, AI, r2, vx, vy, vz);
    out.flx_h[(size_t)0 * fs + off + c] = flux * rarea_ij * dt;
    const T rarea_n = g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + c + 1];
    out.flx_h[(size_t)3 * fs + off + c + 1] = -flux * rarea_n * dt;
    store_xc(AI, XR(ij, AI, 1) - vx * r2 * dt * T(0.5), XR(ij, AI, 2) - vy * r2 * dt * T(0.5),
             XR(ij, AI, 3) - vz * r2 * dt * T(0.5));
  } else {
    out.flx_h[(size_t)0 * fs + off + c] = T(0);
    store_xc(AI, T(0), T(0), T(0));
  }
  // flx_h(ij,4) when no AI face of im1j writes it
  if (!(inJ && i - 1 >= gmin - 1 && i - 1 <= gmax)) out.flx_h[(size_t)3 * fs + off + c] = T(0);
  // AIJ face: flx_h(ij,2), flx_h(ip1jp1,5), GRD_xc(ij,AIJ)   (:261-283)
  if (extI && extJ) {
    T r2, vx, vy, vz;
    const Tri<T> ti = tri_TI_s(D, in, g, l, off, i, j, sgp);
    const Tri<T> tj = tri_TJ(D, in, g, l, off, ij);
    const T flux = face(ti, tj, AIJ, r2, vx, vy, vz);
    out.flx_h[(size_t)1 * fs + off + c] = flux * rarea_ij * dt;
    const T rarea_n = g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + c + G + 1];
    out.flx_h[(size_t)4 * fs + off + c + G + 1] = -flux * rarea_n * dt;
    store_xc(AIJ, XR(ij, AIJ, 1) - vx * r2 * dt * T(0.5), XR(ij, AIJ, 2) - vy * r2 * dt * T(0.5),
             XR(ij, AIJ, 3) - vz * r2 * dt * T(0.5));
  } else {
    out.flx_h[(size_t)1 * fs + off + c] = T(0);
    store_xc(AIJ, T(0), T(0), T(0));
  }
  if (!(i - 1 >= gmin - 1 && i - 1 <= gmax && j - 1 >= gmin - 1 && j - 1 <= gmax))
    out.flx_h[(size_t)4 * fs + off + c] = T(0);
  // AJ face: flx_h(ij,3), flx_h(ijp1,6), GRD_xc(ij,AJ)   (:286-309), singular flx_h(gmin,gmin,6)=0 (:311-320)
  if (inI && extJ) {
    T r2, vx, vy, vz;
    const Tri<T> tj = tri_TJ(D, in, g, l, off, ij);
    const Tri<T> ti = tri_TI_s(D, in, g, l, off, i - 1, j, sgp);
    const T flux = face(tj, ti, AJ, r2, vx, vy, vz);
    out.flx_h[(size_t)2 * fs + off + c] = flux * rarea_ij * dt;
    const T rarea_n = g.GMTR_p[(size_t)(P_RAREA - 1) * gw + (size_t)l * D.gall + c + G];
    const bool sing6 = sgp && i == gmin && j + 1 == gmin;
    out.flx_h[(size_t)5 * fs + off + c + G] = sing6 ? T(0) : -flux * rarea_n * dt;
    store_xc(AJ, XR(ij, AJ, 1) - vx * r2 * dt * T(0.5), XR(ij, AJ, 2) - vy * r2 * dt * T(0.5),
             XR(ij, AJ, 3) - vz * r2 * dt * T(0.5));
  } else {
    out.flx_h[(size_t)2 * fs + off + c] = T(0);
    store_xc(AJ, T(0), T(0), T(0));
  }
  if (!(inI && j - 1 >= gmin - 1 && j - 1 <= gmax)) out.flx_h[(size_t)5 * fs + off + c] = T(0);
}

template <typename T>
__global__ void k_horizontal_flux_pl(Dims D, FluxIn<T> in, FluxOut<T> out, Geo<T> g, T dt) {
  // poles (:326-374): one thread per (k, pole)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.kall * kLallPl) return;
  const int k = t % D.kall, l = t / D.kall;
  const T EPS = Num<T>::eps();
  const size_t off = ((size_t)l * D.kall + k) * kGallPl;
  const size_t fsp = (size_t)kLallPl * D.kall * kGallPl;
  auto GT = [&](int v, int w) { return g.GMTR_t_pl[((size_t)(w - 1) * kLallPl + l) * kGallPl + (v - 1)]; };
  auto GA = [&](int v, int h) { return g.GMTR_a_pl[((size_t)(h - 1) * kLallPl + l) * kGallPl + (v - 1)]; };
  const T rarea = g.GMTR_p_pl[((size_t)(P_RAREA - 1) * kLallPl + l) * kGallPl + 0];
  T rt[7], xt[7], yt[7], zt[7];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v + 1 == 7) ? 2 : v + 1;
    rt[v] = in.rho_pl[off + 0] * GT(v, W1) + in.rho_pl[off + v - 1] * GT(v, W2) + in.rho_pl[off + vp - 1] * GT(v, W3);
    xt[v] = in.rhovx_pl[off + 0] * GT(v, W1) + in.rhovx_pl[off + v - 1] * GT(v, W2) + in.rhovx_pl[off + vp - 1] * GT(v, W3);
    yt[v] = in.rhovy_pl[off + 0] * GT(v, W1) + in.rhovy_pl[off + v - 1] * GT(v, W2) + in.rhovy_pl[off + vp - 1] * GT(v, W3);
    zt[v] = in.rhovz_pl[off + 0] * GT(v, W1) + in.rhovz_pl[off + v - 1] * GT(v, W2) + in.rhovz_pl[off + vp - 1] * GT(v, W3);
  }
  for (int v = 2; v <= 6; ++v) {
    const int vm = (v - 1 == 1) ? 6 : v - 1;
    const T rr = T(1) / mx(rt[vm] + rt[v], EPS);
    const T vx = xt[vm] + xt[v], vy = yt[vm] + yt[v], vz = zt[vm] + zt[v];
    const T flux = T(0.5) * (vx * GA(v, HNX) + vy * GA(v, HNY) + vz * GA(v, HNZ));
    out.flx_h_pl[off + v - 1] = flux * rarea * dt;
    auto XR = [&](int x) { return g.GRD_xr_pl[((size_t)(x - 1) * kLallPl + l) * kGallPl + (v - 1)]; };
    out.GRD_xc_pl[0 * fsp + off + v - 1] = XR(1) - vx * rr * dt * T(0.5);
    out.GRD_xc_pl[1 * fsp + off + v - 1] = XR(2) - vy * rr * dt * T(0.5);
    out.GRD_xc_pl[2 * fsp + off + v - 1] = XR(3) - vz * rr * dt * T(0.5);
  }
}

// ---------------------------------------------------------------------------
// horizontal_limiter_thuburn

// 4-point bounds of face a (AI, AIJ, AJ) of cell c = (i,j) in one (k,l) slab,
// including the index clamps im1j = max(im1j,1), ijm1 = max(ijm1,1) of
// :152-153 and the singular AIJ stencil of :192-214.
template <typename T>
__device__ __forceinline__ void face_bounds(const Dims &D, const T *q, int i, int j, int a, bool sgp,
                                            T &qmin, T &qmax) {
  const int G = D.gall_1d, ij = (j - 1) * G + i;
  const int ip1j = ij + 1, ip1jp1 = ij + G + 1, ijp1 = ij + G;
  int im1j = ij - 1, ijm1 = ij - G;
  if (im1j < 1) im1j = 1;
  if (ijm1 < 1) ijm1 = 1;
  const T q0 = q[ij - 1];
  T b, c, d;
  if (a == AI) {
    b = q[ijm1 - 1], c = q[ip1j - 1], d = q[ip1jp1 - 1];
  } else if (a == AIJ) {
    if (sgp && i == D.gmin - 1 && j == D.gmin - 1) b = q[ip1jp1 - 1], c = q[ij + G + 2 - 1], d = q[ijp1 - 1];
    else b = q[ip1j - 1], c = q[ip1jp1 - 1], d = q[ijp1 - 1];
  } else {
    b = q[ip1jp1 - 1], c = q[ijp1 - 1], d = q[im1j - 1];
  }
  qmin = mn(mn(mn(q0, b), c), d);
  qmax = mx(mx(mx(q0, b), c), d);
}

template <typename T>
__global__ void k_hlim_qout(Dims D, LimIn<T> in, T *Qout) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall;
  const int i = c % D.gall_1d + 1, j = c / D.gall_1d + 1, G = D.gall_1d;
  const size_t off = (size_t)kl * D.gall;
  const size_t fs = (size_t)D.lall * D.kall * D.gall;
  const T *q = in.q + off;
  const T q0 = q[c];
  if (i < D.gmin || i > D.gmax || j < D.gmin || j > D.gmax) {  // halo: Qout = q   (:288-301)
    Qout[0 * fs + off + c] = q0;
    Qout[1 * fs + off + c] = q0;
    return;
  }
  const bool sgp = D.have_sgp[l] != 0;
  const T BIG = Num<T>::big(), EPS = Num<T>::eps();
  auto cm = [&](int cell0, int m) { return in.cmask[(size_t)(m - 1) * fs + off + cell0]; };
  // Qin(ij,.,1..3) from the faces of ij; Qin(ij,.,4..6) from the faces of im1j, im1jm1, ijm1
  T qin_min[7], qin_max[7];
  {
    T lo, hi, cc;
    face_bounds(D, q, i, j, AI, sgp, lo, hi); cc = cm(c, 1);
    qin_min[1] = cc * lo + (T(1) - cc) * BIG; qin_max[1] = cc * hi + (T(1) - cc) * (-BIG);
    face_bounds(D, q, i, j, AIJ, sgp, lo, hi); cc = cm(c, 2);
    qin_min[2] = cc * lo + (T(1) - cc) * BIG; qin_max[2] = cc * hi + (T(1) - cc) * (-BIG);
    face_bounds(D, q, i, j, AJ, sgp, lo, hi); cc = cm(c, 3);
    qin_min[3] = cc * lo + (T(1) - cc) * BIG; qin_max[3] = cc * hi + (T(1) - cc) * (-BIG);
    face_bounds(D, q, i - 1, j, AI, sgp, lo, hi); cc = cm(c - 1, 1);
    qin_min[4] = cc * BIG + (T(1) - cc) * lo; qin_max[4] = cc * (-BIG) + (T(1) - cc) * hi;
    face_bounds(D, q, i - 1, j - 1, AIJ, sgp, lo, hi); cc = cm(c - G - 1, 2);
    qin_min[5] = cc * BIG + (T(1) - cc) * lo; qin_max[5] = cc * (-BIG) + (T(1) - cc) * hi;
    face_bounds(D, q, i, j - 1, AJ, sgp, lo, hi); cc = cm(c - G, 3);
    qin_min[6] = cc * BIG + (T(1) - cc) * lo; qin_max[6] = cc * (-BIG) + (T(1) - cc) * hi;
  }
  T qnext_min = q0, qnext_max = q0;
  for (int f = 1; f <= 6; ++f) qnext_min = mn(qnext_min, qin_min[f]);
  for (int f = 1; f <= 6; ++f) qnext_max = mx(qnext_max, qin_max[f]);
  T ch[7], cmk[7];
  for (int f = 1; f <= 6; ++f) {
    ch[f] = in.ch[(size_t)(f - 1) * fs + off + c];
    cmk[f] = mn(ch[f], T(0));
  }
  const T Cin = cmk[1] + cmk[2] + cmk[3] + cmk[4] + cmk[5] + cmk[6];
  const T Cout = ch[1] - cmk[1] + ch[2] - cmk[2] + ch[3] - cmk[3] + ch[4] - cmk[4] + ch[5] - cmk[5] + ch[6] - cmk[6];
  const T CQmin = cmk[1] * qin_min[1] + cmk[2] * qin_min[2] + cmk[3] * qin_min[3] + cmk[4] * qin_min[4] +
                  cmk[5] * qin_min[5] + cmk[6] * qin_min[6];
  const T CQmax = cmk[1] * qin_max[1] + cmk[2] * qin_max[2] + cmk[3] * qin_max[3] + cmk[4] * qin_max[4] +
                  cmk[5] * qin_max[5] + cmk[6] * qin_max[6];
  const T zerosw = T(0.5) - fsign(T(0.5), fabs(Cout) - EPS);
  const T dv = in.d[off + c];
  Qout[0 * fs + off + c] = (q0 - CQmax - qnext_max * (T(1) - Cin - Cout + dv)) / (Cout + zerosw) * (T(1) - zerosw) + q0 * zerosw;
  Qout[1 * fs + off + c] = (q0 - CQmin - qnext_min * (T(1) - Cin - Cout + dv)) / (Cout + zerosw) * (T(1) - zerosw) + q0 * zerosw;
}

template <typename T>
__global__ void k_hlim_qout_pl(Dims D, LimIn<T> in, T *Qout_pl, T *Qin_pl) {
  // (:307-367): Qout_pl(n) from the 5 ring faces; Qout_pl(2:6) = 0; keep Qin_pl for the apply
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.kall * kLallPl) return;
  const int k = t % D.kall, l = t / D.kall;
  const T BIG = Num<T>::big(), EPS = Num<T>::eps();
  const size_t off = ((size_t)l * D.kall + k) * kGallPl;
  const size_t fsp = (size_t)kLallPl * D.kall * kGallPl;
  const T *q = in.q_pl + off;
  T qmin1[7], qmax1[7];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v + 1 == 7) ? 2 : v + 1, vm = (v - 1 == 1) ? 6 : v - 1;
    const T lo = mn(mn(mn(q[0], q[v - 1]), q[vm - 1]), q[vp - 1]);
    const T hi = mx(mx(mx(q[0], q[v - 1]), q[vm - 1]), q[vp - 1]);
    const T c = in.cmask_pl[off + v - 1];
    qmin1[v] = c * lo + (T(1) - c) * BIG;
    qmax1[v] = c * hi + (T(1) - c) * (-BIG);
    // Qin_pl(v,k,l,min/max,1/2)
    Qin_pl[((size_t)0 * 2 + 0) * fsp + off + v - 1] = qmin1[v];
    Qin_pl[((size_t)0 * 2 + 1) * fsp + off + v - 1] = c * BIG + (T(1) - c) * lo;
    Qin_pl[((size_t)1 * 2 + 0) * fsp + off + v - 1] = qmax1[v];
    Qin_pl[((size_t)1 * 2 + 1) * fsp + off + v - 1] = c * (-BIG) + (T(1) - c) * hi;
  }
  T qnmin = q[0], qnmax = q[0];
  for (int v = 2; v <= 6; ++v) {
    qnmin = mn(qnmin, qmin1[v]);
    qnmax = mx(qnmax, qmax1[v]);
  }
  T Cin = 0, Cout = 0, CQmax = 0, CQmin = 0;
  for (int v = 2; v <= 6; ++v) {
    const T chm = in.cmask_pl[off + v - 1] * in.ch_pl[off + v - 1];
    Cin = Cin + chm;
    Cout = Cout - chm + in.ch_pl[off + v - 1];
    CQmin = CQmin + chm * qmin1[v];
    CQmax = CQmax + chm * qmax1[v];
  }
  const T zerosw = T(0.5) - fsign(T(0.5), fabs(Cout) - EPS);
  const T qn = q[0], dn = in.d_pl[off];
  Qout_pl[0 * fsp + off] = (qn - CQmax - qnmax * (T(1) - Cin - Cout + dn)) / (Cout + zerosw) * (T(1) - zerosw) + qn * zerosw;
  Qout_pl[1 * fsp + off] = (qn - CQmin - qnmin * (T(1) - Cin - Cout + dn)) / (Cout + zerosw) * (T(1) - zerosw) + qn * zerosw;
  for (int v = 2; v <= 6; ++v) {
    Qout_pl[0 * fsp + off + v - 1] = T(0);
    Qout_pl[1 * fsp + off + v - 1] = T(0);
  }
}

template <typename T>
__global__ void k_hlim_apply(Dims D, LimIn<T> in, T *q_a, const T *Qout) {
  // (:378-410): cells (i,j) in [gmin-1,gmax]^2, faces 1..3, mirrored to 4..6
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.gall) return;
  const int kl = blockIdx.y, l = kl / D.kall;
  const int i = c % D.gall_1d + 1, j = c / D.gall_1d + 1, G = D.gall_1d;
  if (i < D.gmin - 1 || i > D.gmax || j < D.gmin - 1 || j > D.gmax) return;
  const size_t off = (size_t)kl * D.gall;
  const size_t fs = (size_t)D.lall * D.kall * D.gall;
  const bool sgp = D.have_sgp[l] != 0;
  const T BIG = Num<T>::big();
  const T *q = in.q + off;
  const int nbs[4] = {0, c + 1, c + G + 1, c + G};
  const int faces[4] = {0, AI, AIJ, AJ};
  for (int m = 1; m <= 3; ++m) {
    const int nb = nbs[m];
    T lo, hi;
    face_bounds(D, q, i, j, faces[m], sgp, lo, hi);
    const T cc = in.cmask[(size_t)(m - 1) * fs + off + c];
    const T own_min = cc * lo + (T(1) - cc) * BIG, own_max = cc * hi + (T(1) - cc) * (-BIG);
    const T nb_min = cc * BIG + (T(1) - cc) * lo, nb_max = cc * (-BIG) + (T(1) - cc) * hi;
    T v = q_a[(size_t)(m - 1) * fs + off + c];
    v = cc * mn(mx(v, own_min), own_max) + (T(1) - cc) * mn(mx(v, nb_min), nb_max);
    const T on_max = Qout[1 * fs + off + nb], on_min = Qout[0 * fs + off + nb];
    const T os_max = Qout[1 * fs + off + c], os_min = Qout[0 * fs + off + c];
    v = cc * mx(mn(v, on_max), on_min) + (T(1) - cc) * mx(mn(v, os_max), os_min);
    q_a[(size_t)(m - 1) * fs + off + c] = v;
    q_a[(size_t)(m + 2) * fs + off + nb] = v;
  }
}

template <typename T>
__global__ void k_hlim_apply_pl(Dims D, LimIn<T> in, T *q_a_pl, const T *Qout_pl, const T *Qin_pl) {
  // (:412-425)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.kall * kLallPl * 5) return;
  const int v = t % 5 + 2, kl = t / 5;
  const size_t off = (size_t)kl * kGallPl;
  const size_t fsp = (size_t)kLallPl * D.kall * kGallPl;
  const T c = in.cmask_pl[off + v - 1];
  T x = q_a_pl[off + v - 1];
  const T i1min = Qin_pl[((size_t)0 * 2 + 0) * fsp + off + v - 1], i2min = Qin_pl[((size_t)0 * 2 + 1) * fsp + off + v - 1];
  const T i1max = Qin_pl[((size_t)1 * 2 + 0) * fsp + off + v - 1], i2max = Qin_pl[((size_t)1 * 2 + 1) * fsp + off + v - 1];
  x = c * mn(mx(x, i1min), i1max) + (T(1) - c) * mn(mx(x, i2min), i2max);
  x = c * mx(mn(x, Qout_pl[1 * fsp + off + v - 1]), Qout_pl[0 * fsp + off + v - 1]) +
      (T(1) - c) * mx(mn(x, Qout_pl[1 * fsp + off + 0]), Qout_pl[0 * fsp + off + 0]);
  q_a_pl[off + v - 1] = x;
}

// ---------------------------------------------------------------------------
// vertical_limiter_thuburn: one thread per column g, the k-recurrence in registers
template <typename T, bool POLE>
__device__ __forceinline__ void vlim_qout(const T *q, const T *d, const T *ck1, const T *ck2, size_t s, int k,
                                          T &inflagL, T &Qmin, T &Qmax) {
  const T BIG = Num<T>::big(), EPS = Num<T>::eps();
  inflagL = T(0.5) - fsign(T(0.5), ck1[(size_t)k * s]);
  const T inflagU = T(0.5) + fsign(T(0.5), ck1[(size_t)(k + 1) * s]);
  const T qk = q[(size_t)k * s], qm = q[(size_t)(k - 1) * s], qp = q[(size_t)(k + 1) * s];
  const T minL = mn(qk, qm) + (T(1) - inflagL) * BIG;
  const T minU = mn(qk, qp) + (T(1) - inflagU) * BIG;
  const T maxL = mx(qk, qm) - (T(1) - inflagL) * BIG;
  const T maxU = mx(qk, qp) - (T(1) - inflagU) * BIG;
  const T qnmin = mn(mn(minL, minU), qk);
  const T qnmax = mx(mx(maxL, maxU), qk);
  const T c1 = ck1[(size_t)k * s], c2 = ck2[(size_t)k * s];
  const T Cin = inflagL * c1 + inflagU * c2;
  const T Cout = (T(1) - inflagL) * c1 + (T(1) - inflagU) * c2;
  T CQmin, CQmax;
  if (POLE) {  // the pole loop groups ck*Qin first (:212-215)
    CQmax = inflagL * (c1 * maxL) + inflagU * (c2 * maxU);
    CQmin = inflagL * (c1 * minL) + inflagU * (c2 * minU);
  } else {
    CQmin = inflagL * c1 * minL + inflagU * c2 * minU;
    CQmax = inflagL * c1 * maxL + inflagU * c2 * maxU;
  }
  const T zerosw = T(0.5) - fsign(T(0.5), fabs(Cout) - EPS);
  const T dv = d[(size_t)k * s];
  Qmin = ((qk - qnmax) + qnmax * (Cin + Cout - dv) - CQmax) / (Cout + zerosw) * (T(1) - zerosw) + qk * zerosw;
  Qmax = ((qk - qnmin) + qnmin * (Cin + Cout - dv) - CQmin) / (Cout + zerosw) * (T(1) - zerosw) + qk * zerosw;
}

template <typename T, bool POLE>
__global__ void k_vlim(int ncol, int colsize, int kall, int kmin, int kmax, T *q_h, const T *q, const T *d,
                       const T *ck) {
  // column index t -> (l, g); fields (g,k,l) with stride colsize between levels
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncol) return;
  const int l = t / colsize, g = t % colsize;
  const size_t base = (size_t)l * kall * colsize + g;
  const size_t ck2off = (size_t)(ncol / colsize) * kall * colsize;
  const T *ck1 = ck + base, *ck2 = ck + ck2off + base;
  T fl, Qmin_km1, Qmax_km1;
  vlim_qout<T, POLE>(q + base, d + base, ck1, ck2, colsize, kmin - 1, fl, Qmin_km1, Qmax_km1);
  for (int k = kmin; k <= kmax - 1; ++k) {  // 0-based k = Fortran kmin+1 .. kmax
    T inflagL, Qmin, Qmax;
    vlim_qout<T, POLE>(q + base, d + base, ck1, ck2, colsize, k, inflagL, Qmin, Qmax);
    const size_t e = base + (size_t)k * colsize;
    const T qh = q_h[e];
    q_h[e] = inflagL * mx(mn(qh, Qmax_km1), Qmin_km1) + (T(1) - inflagL) * mx(mn(qh, Qmax), Qmin);
    Qmin_km1 = Qmin;
    Qmax_km1 = Qmax;
  }
}

// ---------------------------------------------------------------------------
// halo/pole fill as one gather: var(dst) = var(src) for every (entry, k, v)
template <typename T>
__global__ void k_gather(int nent, const int *__restrict__ dst, const int *__restrict__ src, int npt_rgn, int gall,
                         int lall, int kmax, int vmax, T *var, T *var_pl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nent * kmax * vmax;
  if (t >= total) return;
  const int e = (int)(t % nent);
  const int kv = (int)(t / nent);
  const int k = kv % kmax, v = kv / kmax;
  auto addr = [&](int p) -> T * {
    if (p < npt_rgn) {
      const int l = p / gall, ij0 = p % gall;
      return var + (((size_t)v * lall + l) * kmax + k) * gall + ij0;
    }
    const int qd = p - npt_rgn, lp = qd / kGallPl, vv = qd % kGallPl;
    return var_pl + (((size_t)v * kLallPl + lp) * kmax + k) * kGallPl + vv;
  };
  *addr(dst[e]) = *addr(src[e]);
}

// ---------------------------------------------------------------------------
// launchers
static inline dim3 slab_grid(const Dims &D, int threads) {
  return dim3((D.gall + threads - 1) / threads, D.kall * D.lall);
}

template <typename T>
void launch_horizontal_flux(const Dims &D, const FluxIn<T> &in, const FluxOut<T> &out, const Geo<T> &g, T dt,
                            cudaStream_t s) {
  k_horizontal_flux<T><<<slab_grid(D, 128), 128, 0, s>>>(D, in, out, g, dt);
  if (D.have_pl) k_horizontal_flux_pl<T><<<(D.kall * kLallPl + 63) / 64, 64, 0, s>>>(D, in, out, g, dt);
}

template <typename T>
void launch_hlim_qout(const Dims &D, const LimIn<T> &in, T *Qout, T *Qout_pl, T *Qin_pl, cudaStream_t s) {
  k_hlim_qout<T><<<slab_grid(D, 128), 128, 0, s>>>(D, in, Qout);
  if (D.have_pl) k_hlim_qout_pl<T><<<(D.kall * kLallPl + 63) / 64, 64, 0, s>>>(D, in, Qout_pl, Qin_pl);
}

template <typename T>
void launch_hlim_apply(const Dims &D, const LimIn<T> &in, T *q_a, T *q_a_pl, const T *Qout, const T *Qout_pl,
                       const T *Qin_pl, cudaStream_t s) {
  k_hlim_apply<T><<<slab_grid(D, 128), 128, 0, s>>>(D, in, q_a, Qout);
  if (D.have_pl) k_hlim_apply_pl<T><<<(D.kall * kLallPl * 5 + 63) / 64, 64, 0, s>>>(D, in, q_a_pl, Qout_pl, Qin_pl);
}

template <typename T>
void launch_vlim(const Dims &D, T *q_h, T *q_h_pl, const T *q, const T *q_pl, const T *d, const T *d_pl,
                 const T *ck, const T *ck_pl, cudaStream_t s) {
  if (D.kmax <= D.kmin) return;
  const int ncol = D.gall * D.lall;
  k_vlim<T, false><<<(ncol + 127) / 128, 128, 0, s>>>(ncol, D.gall, D.kall, D.kmin, D.kmax, q_h, q, d, ck);
  const int ncp = kGallPl * kLallPl;
  if (D.have_pl) k_vlim<T, true><<<1, 32, 0, s>>>(ncp, kGallPl, D.kall, D.kmin, D.kmax, q_h_pl, q_pl, d_pl, ck_pl);
}

template <typename T>
void launch_gather(const Dims &D, int nent, const int *dst, const int *src, int kmax, int vmax, T *var, T *var_pl,
                   cudaStream_t s) {
  const long long total = (long long)nent * kmax * vmax;
  if (total == 0) return;
  const int threads = 256;
  const long long blocks = (total + threads - 1) / threads;
  k_gather<T><<<(unsigned)blocks, threads, 0, s>>>(nent, dst, src, D.gall * D.lall, D.gall, D.lall, kmax, vmax, var,
                                                   var_pl);
}

#define INSTANTIATE(T)                                                                                        \
  template void launch_horizontal_flux<T>(const Dims &, const FluxIn<T> &, const FluxOut<T> &, const Geo<T> &, \
                                          T, cudaStream_t);                                                   \
  template void launch_hlim_qout<T>(const Dims &, const LimIn<T> &, T *, T *, T *, cudaStream_t);             \
  template void launch_hlim_apply<T>(const Dims &, const LimIn<T> &, T *, T *, const T *, const T *,          \
                                     const T *, cudaStream_t);                                                \
  template void launch_vlim<T>(const Dims &, T *, T *, const T *, const T *, const T *, const T *, const T *, \
                               const T *, cudaStream_t);                                                      \
  template void launch_gather<T>(const Dims &, int, const int *, const int *, int, int, T *, T *, cudaStream_t);
INSTANTIATE(double)
INSTANTIATE(float)

}  // namespace icoadv
