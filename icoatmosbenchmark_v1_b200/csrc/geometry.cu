// The grid and its metrics built on the device: the setup of dyn_metrics (GMTR_p/t/a_setup,
// kernels/NICAM/dyn_metrics/src/mod_gmtr.f90:46-741, and OPRT_gradient_setup,
// dyn_metrics/src/mod_oprt.f90:499-734) for the synthetic icosahedral grid of this library,
// whose cell positions come from recursive bisection of the icosahedron's ten diamonds
// (the reference reads its positions from a snapshot instead).  Compiled without FMA
// contraction, so every sum and product rounds as in the host build of the same grid
// (icoatmosbenchmark_v1_b200/grid.py); atan2, sin and cos are CUDA's, which can differ from
// the host's by an ulp, so the two builds agree to rounding, not bit for bit.
//
// Layouts are the library's (Fortran column-major = C reversed): GRD_x (3, lall, gall),
// GRD_xr (3 xyz, 3 arcs, lall, gall), GMTR_p (8, lall, gall), GMTR_t (5, 2, lall, gall),
// GMTR_a (12, 3, lall, gall), coef_grad (lall, 3, 7, gall); poles (m, 2, 6), GMTR_a_pl
// (18, 2, 6), coef_grad_pl (2, 3, 6).  Indices below are 0-based: cell (j, i) of a region
// is ij = j * G + i, the interior is [1, G-2]^2.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "capi_internal.h"

namespace icoadv {

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 scl3(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double norm3(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 unit3(D3 a) {
  const double n = norm3(a);
  return {a.x / n, a.y / n, a.z / n};
}
// solid angle of the spherical triangle with unit corners a, b, c (Van Oosterom & Strackee 1983)
__device__ __forceinline__ double tri_area(D3 a, D3 b, D3 c) {
  const double num = fabs(dot3(a, cross3(b, c)));
  const double den = 1.0 + dot3(a, b) + dot3(b, c) + dot3(c, a);
  return 2.0 * atan2(num, den);
}
// angle between unit vectors, robust for small angles
__device__ __forceinline__ double arc_angle(D3 a, D3 b) { return atan2(norm3(cross3(a, b)), dot3(a, b)); }

// array (m, lall, gall) of D3 spread over three planes of `plane` elements
__device__ __forceinline__ D3 ld3(const double *a, size_t plane, size_t o) { return {a[o], a[plane + o], a[2 * plane + o]}; }
__device__ __forceinline__ void st3(double *a, size_t plane, size_t o, D3 v) {
  a[o] = v.x, a[plane + o] = v.y, a[2 * plane + o] = v.z;
}

// ---- positions: the ten diamonds' lattices (n+1)^2 points each, [d][a][b] with a along
// W->S and b along W->N, refined level by level: a new point is the normalised sum of the
// two coarse points it bisects (along a, along b, or along the a = b diagonal)
__global__ void k_geo_lattice_corners(double *lat, int n, const double *corners) {
  const int d = threadIdx.x;
  if (d >= 10) return;
  const size_t N1 = (size_t)n + 1, base = (size_t)d * N1 * N1 * 3;
  const int ca[4] = {0, n, n, 0}, cb[4] = {0, 0, n, n};  // W, S, E, N
  for (int c = 0; c < 4; ++c)
    for (int x = 0; x < 3; ++x) lat[base + ((size_t)ca[c] * N1 + cb[c]) * 3 + x] = corners[(d * 4 + c) * 3 + x];
}
__global__ void k_geo_lattice_level(double *lat, int n, int h) {
  const int g = h / 2, m = n / g + 1;  // points of this level's spacing per side
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10LL * m * m) return;
  const int d = (int)(t / ((long long)m * m)), r = (int)(t % ((long long)m * m));
  const int a = (r / m) * g, b = (r % m) * g;
  const bool ah = a % h == 0, bh = b % h == 0;
  if (ah && bh) return;  // a coarse point
  const size_t N1 = (size_t)n + 1, base = (size_t)d * N1 * N1 * 3;
  auto P = [&](int aa, int bb) {
    const size_t o = base + ((size_t)aa * N1 + bb) * 3;
    return D3{lat[o], lat[o + 1], lat[o + 2]};
  };
  D3 v;
  if (!ah && bh) v = unit3(add3(P(a - g, b), P(a + g, b)));
  else if (ah && !bh) v = unit3(add3(P(a, b - g), P(a, b + g)));
  else v = unit3(add3(P(a - g, b - g), P(a + g, b + g)));
  const size_t o = base + ((size_t)a * N1 + b) * 3;
  lat[o] = v.x, lat[o + 1] = v.y, lat[o + 2] = v.z;
}
// interior cells of every region from its diamond's lattice (unit vectors), halo zero; poles
__global__ void k_geo_positions(const double *lat, int n_dia, int rl1, int nmax, int G, int lall, double *xu,
                                double *xu_pl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall;
  if (t == 0) {
    for (int q = 0; q < 3 * kLallPl * kGallPl; ++q) xu_pl[q] = 0.0;
    xu_pl[(size_t)2 * kLallPl * kGallPl + 0] = 1.0;         // z of the north pole centre
    xu_pl[(size_t)2 * kLallPl * kGallPl + kGallPl] = -1.0;  // z of the south pole centre
  }
  if (t >= (long long)plane) return;
  const int r = (int)(t / gall), c = (int)(t % gall), j = c / G, i = c % G;
  D3 v = {0.0, 0.0, 0.0};
  if (i >= 1 && i <= G - 2 && j >= 1 && j <= G - 2) {
    const int d = r / (rl1 * rl1), rem = r % (rl1 * rl1), jr = rem / rl1, ir = rem % rl1;
    const int a = ir * nmax + (i - 1), b = jr * nmax + (j - 1);
    const size_t N1 = (size_t)n_dia + 1, o = (size_t)d * N1 * N1 * 3 + ((size_t)a * N1 + b) * 3;
    v = {lat[o], lat[o + 1], lat[o + 2]};
  }
  st3(xu, plane, (size_t)t, v);
}
__global__ void k_geo_scale(const double *xu, const double *xu_pl, size_t n, double R, double *out, double *out_pl) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = xu[t] * R;
  if (t < (size_t)3 * kLallPl * kGallPl) out_pl[t] = xu_pl[t] * R;
}

// ---- triangle centres (unit) and GMTR_t of TI = (ij, ip1j, ip1jp1), TJ = (ij, ip1jp1, ijp1)
// for (j, i) in [0, G-2]^2; xt is (2 TI/TJ, 3 xyz, lall, gall)
__global__ void k_geo_tri(const double *xu, int G, int lall, double R, double *xt, double *gt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall;
  if (t >= (long long)plane) return;
  const int c = (int)(t % gall), j = c / G, i = c % G;
  const size_t o = (size_t)t;
  for (int tt = 0; tt < 2; ++tt) {
    D3 ct = {0.0, 0.0, 0.0};
    double w[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (i <= G - 2 && j <= G - 2) {
      const D3 vij = ld3(xu, plane, o), vip1j = ld3(xu, plane, o + 1), vip1jp1 = ld3(xu, plane, o + G + 1),
               vijp1 = ld3(xu, plane, o + G);
      const D3 v0 = vij, v1 = tt == 0 ? vip1j : vip1jp1, v2 = tt == 0 ? vip1jp1 : vijp1;
      ct = unit3(add3(add3(v0, v1), v2));
      const double a1 = tri_area(ct, v1, v2), a2 = tri_area(ct, v2, v0), a3 = tri_area(ct, v0, v1);
      const double area = a1 + a2 + a3;
      w[0] = area * R * R;
      w[1] = 1.0 / (area * R * R);
      w[2] = a1 / area, w[3] = a2 / area, w[4] = a3 / area;
    }
    st3(xt + (size_t)tt * 3 * plane, plane, o, ct);
    for (int q = 0; q < 5; ++q) gt[((size_t)q * 2 + tt) * plane + o] = w[q];
  }
}
// unused triangles and the pentagon (mod_gmtr.f90:293-299): one thread per region
__global__ void k_geo_tri_fix(int G, int lall, const int *have_sgp, double *xt, double *gt) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= lall) return;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall, lo = (size_t)l * gall;
  auto copy = [&](int tdst, size_t odst, int tsrc, size_t osrc) {
    for (int q = 0; q < 5; ++q) gt[((size_t)q * 2 + tdst) * plane + odst] = gt[((size_t)q * 2 + tsrc) * plane + osrc];
    for (int x = 0; x < 3; ++x)
      xt[((size_t)tdst * 3 + x) * plane + odst] = xt[((size_t)tsrc * 3 + x) * plane + osrc];
  };
  copy(0, lo + (size_t)0 * G + (G - 2), 1, lo + (size_t)0 * G + (G - 2));  // TI(j=0, i=G-2) = TJ
  copy(1, lo + (size_t)(G - 2) * G + 0, 0, lo + (size_t)(G - 2) * G + 0);  // TJ(j=G-2, i=0) = TI
  if (have_sgp[l]) copy(0, lo + 0, 1, lo + 1);                             // TI(0,0) = TJ(0,1)
}

// ---- hexagon arcs (mod_gmtr.f90:566-676): GMTR_a (HN x/y/z, HT x/y/z scaled by the arc
// length) and the arc midpoints GRD_xr.  AI runs from xt(ij,TI) to xt(ijm1,TJ), AIJ from
// xt(ij,TJ) to xt(ij,TI), AJ from xt(im1j,TI) to xt(ij,TJ), with the unused-arc and pentagon
// choices of the reference.
__global__ void k_geo_arc(const double *xt, int G, int lall, const int *have_sgp, double R, double *ga,
                          double *xr) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall;
  if (t >= 3LL * (long long)plane) return;
  const int a = (int)(t / plane);
  const size_t o = (size_t)(t % plane);
  const int l = (int)(o / gall), c = (int)(o % gall), j = c / G, i = c % G;
  auto X = [&](int tt, int jj, int ii) { return ld3(xt + (size_t)tt * 3 * plane, plane, (size_t)l * gall + (size_t)jj * G + ii); };
  const D3 z = {0.0, 0.0, 0.0};
  D3 f = z, to = z;
  if (a == 0) {
    if (j >= 1 && j <= G - 2 && i <= G - 2) f = X(0, j, i), to = X(1, j - 1, i);
  } else if (a == 1) {
    if (j <= G - 2 && i <= G - 2) f = X(1, j, i), to = X(0, j, i);
    if (j == 0 && i == G - 2) f = X(1, 0, G - 2), to = X(0, 1, G - 2);
    if (j == G - 2 && i == 0) f = X(1, G - 2, 1), to = X(0, G - 2, 0);
  } else {
    if (j <= G - 2 && i >= 1 && i <= G - 2) f = X(0, j, i - 1), to = X(1, j, i);
    if (have_sgp[l] && j == 0 && i == 1) f = X(0, 1, 1), to = X(1, 0, 1);
  }
  const bool ok = norm3(f) > 0.0 && norm3(to) > 0.0;
  double hn[3] = {0.0, 0.0, 0.0}, ht[3] = {0.0, 0.0, 0.0};
  D3 mid = z;
  if (ok) {
    const double dist = arc_angle(f, to) * R;
    const D3 nv = cross3(f, to), tv = sub3(to, f);
    const double nl = norm3(nv), tl = norm3(tv);
    if (nl > 0.0) hn[0] = nv.x * (dist / nl), hn[1] = nv.y * (dist / nl), hn[2] = nv.z * (dist / nl);
    if (tl > 0.0) ht[0] = tv.x * (dist / tl), ht[1] = tv.y * (dist / tl), ht[2] = tv.z * (dist / tl);
    mid = scl3(unit3(add3(f, to)), R);
  }
  for (int x = 0; x < 3; ++x) {
    ga[((size_t)x * 3 + a) * plane + o] = hn[x];
    ga[((size_t)(3 + x) * 3 + a) * plane + o] = ht[x];
  }
  for (int q = 6; q < 12; ++q) ga[((size_t)q * 3 + a) * plane + o] = 0.0;
  xr[((size_t)0 * 3 + a) * plane + o] = mid.x;
  xr[((size_t)1 * 3 + a) * plane + o] = mid.y;
  xr[((size_t)2 * 3 + a) * plane + o] = mid.z;
}

// ---- cell areas (mod_gmtr.f90:101-152: the 6 triangles around the cell, pentagon vertex 6 =
// vertex 1) of interior cells, and the local frame entries of every point
__global__ void k_geo_area(const double *xu, const double *xt, int G, int lall, const int *have_sgp, double R,
                           double *gp) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall;
  if (t >= (long long)plane) return;
  const size_t o = (size_t)t;
  const int l = (int)(o / gall), c = (int)(o % gall), j = c / G, i = c % G;
  const D3 X = ld3(xu, plane, o);
  double area = 0.0, rarea = 0.0;
  if (i >= 1 && i <= G - 2 && j >= 1 && j <= G - 2) {
    auto T = [&](int tt, int jj, int ii) { return ld3(xt + (size_t)tt * 3 * plane, plane, (size_t)l * gall + (size_t)jj * G + ii); };
    D3 w[7] = {T(1, j - 1, i), T(0, j, i), T(1, j, i), T(0, j, i - 1), T(1, j - 1, i - 1), T(0, j - 1, i - 1), {}};
    if (have_sgp[l] && j == 1 && i == 1) w[5] = w[0];
    w[6] = w[0];
    double s = 0.0;
    for (int v = 0; v < 6; ++v) s = s + tri_area(X, w[v], w[v + 1]);
    area = s * R * R;
    rarea = 1.0 / area;
  }
  const double lon = atan2(X.y, X.x), sl = sin(lon), cl = cos(lon);
  const double v[8] = {area, rarea, -sl, cl, 0.0, -X.z * cl, -X.z * sl, X.x * cl + X.y * sl};
  for (int q = 0; q < 8; ++q) gp[(size_t)q * plane + o] = v[q];
}

// ---- gradient coefficients (mod_oprt.f90:499-734), interior cells; the pentagon's
// coefficients 0, 1, 5, 6 take the pentagon form
__global__ void k_geo_grad(const double *gt, const double *ga, const double *gp, int G, int lall,
                           const int *have_sgp, double *cg) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gall = (size_t)G * G, plane = (size_t)lall * gall;
  if (t >= 3LL * (long long)plane) return;
  const int d = (int)(t / plane);
  const size_t o = (size_t)(t % plane);
  const int l = (int)(o / gall), c = (int)(o % gall), j = c / G, i = c % G;
  if (!(i >= 1 && i <= G - 2 && j >= 1 && j <= G - 2)) return;
  const size_t ij = o, im1j = o - 1, im1jm1 = o - G - 1, ijm1 = o - G;
  enum { TI = 0, TJ = 1, W1 = 2, W2 = 3, W3 = 4, AI = 0, AIJ = 1, AJ = 2 };
  auto T = [&](size_t p, int tt, int w) { return gt[((size_t)w * 2 + tt) * plane + p]; };
  auto A = [&](size_t p, int a) { return ga[((size_t)d * 3 + a) * plane + p]; };
  const double f = 0.5 * gp[plane + o];
  double cn[7];
  cn[0] = (T(ij, TI, W1) * A(ij, AI) + T(ij, TI, W1) * A(ij, AIJ) + T(ij, TJ, W1) * A(ij, AIJ) +
           T(ij, TJ, W1) * A(ij, AJ) + T(im1j, TI, W2) * A(ij, AJ) - T(im1j, TI, W2) * A(im1j, AI) -
           T(im1jm1, TJ, W2) * A(im1j, AI) - T(im1jm1, TI, W3) * A(im1jm1, AIJ) -
           T(im1jm1, TJ, W2) * A(im1jm1, AIJ) - T(im1jm1, TI, W3) * A(ijm1, AJ) - T(ijm1, TJ, W3) * A(ijm1, AJ) +
           T(ijm1, TJ, W3) * A(ij, AI) - 2 * A(ij, AIJ) - 2 * A(ij, AJ) + 2 * A(im1j, AI) + 2 * A(im1jm1, AIJ) +
           2 * A(ijm1, AJ) - 2 * A(ij, AI)) *
          f;
  cn[1] = (-T(ijm1, TJ, W2) * A(ijm1, AJ) + T(ijm1, TJ, W2) * A(ij, AI) + T(ij, TI, W2) * A(ij, AI) +
           T(ij, TI, W2) * A(ij, AIJ)) *
          f;
  cn[2] = (T(ij, TI, W3) * A(ij, AI) + T(ij, TI, W3) * A(ij, AIJ) + T(ij, TJ, W2) * A(ij, AIJ) +
           T(ij, TJ, W2) * A(ij, AJ)) *
          f;
  cn[3] = (T(ij, TJ, W3) * A(ij, AIJ) + T(ij, TJ, W3) * A(ij, AJ) + T(im1j, TI, W3) * A(ij, AJ) -
           T(im1j, TI, W3) * A(im1j, AI)) *
          f;
  cn[4] = (T(im1j, TI, W1) * A(ij, AJ) - T(im1j, TI, W1) * A(im1j, AI) - T(im1jm1, TJ, W3) * A(im1j, AI) -
           T(im1jm1, TJ, W3) * A(im1jm1, AIJ)) *
          f;
  cn[5] = (-T(im1jm1, TJ, W1) * A(im1j, AI) - T(im1jm1, TJ, W1) * A(im1jm1, AIJ) -
           T(im1jm1, TI, W1) * A(im1jm1, AIJ) - T(im1jm1, TI, W1) * A(ijm1, AJ)) *
          f;
  cn[6] = (-T(im1jm1, TI, W2) * A(im1jm1, AIJ) - T(im1jm1, TI, W2) * A(ijm1, AJ) - T(ijm1, TJ, W1) * A(ijm1, AJ) +
           T(ijm1, TJ, W1) * A(ij, AI)) *
          f;
  if (have_sgp[l] && j == 1 && i == 1) {  // pentagon at (gmin, gmin)
    cn[0] = (T(ij, TI, W1) * A(ij, AI) + T(ij, TI, W1) * A(ij, AIJ) + T(ij, TJ, W1) * A(ij, AIJ) +
             T(ij, TJ, W1) * A(ij, AJ) + T(im1j, TI, W2) * A(ij, AJ) - T(im1j, TI, W2) * A(im1j, AI) -
             T(im1jm1, TJ, W2) * A(im1j, AI) - T(im1jm1, TJ, W2) * A(im1jm1, AIJ) -
             T(ijm1, TJ, W3) * A(im1jm1, AIJ) + T(ijm1, TJ, W3) * A(ij, AI) - 2 * A(ij, AIJ) - 2 * A(ij, AJ) +
             2 * A(im1j, AI) + 2 * A(im1jm1, AIJ) - 2 * A(ij, AI)) *
            f;
    cn[1] = (-T(ijm1, TJ, W2) * A(im1jm1, AIJ) + T(ijm1, TJ, W2) * A(ij, AI) + T(ij, TI, W2) * A(ij, AI) +
             T(ij, TI, W2) * A(ij, AIJ)) *
            f;
    cn[5] = (-T(im1jm1, TJ, W1) * A(im1j, AI) - T(im1jm1, TJ, W1) * A(im1jm1, AIJ)) * f;
    cn[6] = (-T(ijm1, TJ, W1) * A(im1jm1, AIJ) + T(ijm1, TJ, W1) * A(ij, AI)) * f;
  }
  for (int n = 0; n < 7; ++n) cg[(((size_t)l * 3 + d) * 7 + n) * gall + c] = cn[n];
}

// ---- the two pole regions (mod_gmtr.f90 pole sections, mod_oprt.f90:705-731): one thread each
__global__ void k_geo_poles(const double *xu_pl, double R, double *xr_pl, double *gp_pl, double *gt_pl,
                            double *ga_pl, double *cg_pl) {
  const int p = threadIdx.x;
  if (p >= kLallPl) return;
  const size_t PL = (size_t)kLallPl * kGallPl;
  auto X = [&](int v) { return D3{xu_pl[0 * PL + p * kGallPl + v], xu_pl[1 * PL + p * kGallPl + v], xu_pl[2 * PL + p * kGallPl + v]}; };
  auto at = [&](double *a, int m, int v) -> double & { return a[(size_t)m * PL + p * kGallPl + v]; };
  for (int m = 0; m < 3; ++m)
    for (int v = 0; v < kGallPl; ++v) at(xr_pl, m, v) = 0.0;
  for (int m = 0; m < 8; ++m)
    for (int v = 0; v < kGallPl; ++v) at(gp_pl, m, v) = 0.0;
  for (int m = 0; m < 5; ++m)
    for (int v = 0; v < kGallPl; ++v) at(gt_pl, m, v) = 0.0;
  for (int m = 0; m < 18; ++m)
    for (int v = 0; v < kGallPl; ++v) at(ga_pl, m, v) = 0.0;
  D3 xt[kGallPl];
  xt[0] = {0.0, 0.0, 0.0};
  const D3 c0 = X(0);
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    xt[v - 1] = unit3(add3(add3(c0, X(v - 1)), X(vp - 1)));
  }
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    const D3 c = xt[v - 1];
    const double a1 = tri_area(c, X(v - 1), X(vp - 1)), a2 = tri_area(c, X(vp - 1), c0), a3 = tri_area(c, c0, X(v - 1));
    const double ar = a1 + a2 + a3;
    at(gt_pl, 0, v - 1) = ar * R * R;
    at(gt_pl, 1, v - 1) = 1.0 / (ar * R * R);
    at(gt_pl, 2, v - 1) = a1 / ar, at(gt_pl, 3, v - 1) = a2 / ar, at(gt_pl, 4, v - 1) = a3 / ar;
  }
  for (int v = 2; v <= 6; ++v) {
    const int vm = (v == 2) ? 6 : v - 1;
    const D3 f = xt[vm - 1], t = xt[v - 1];
    const double dist = arc_angle(f, t) * R;
    const D3 nv = cross3(f, t), tv = sub3(t, f);
    const double nl = norm3(nv), tl = norm3(tv);
    at(ga_pl, 0, v - 1) = nv.x * dist / nl, at(ga_pl, 1, v - 1) = nv.y * dist / nl, at(ga_pl, 2, v - 1) = nv.z * dist / nl;
    at(ga_pl, 3, v - 1) = tv.x * dist / tl, at(ga_pl, 4, v - 1) = tv.y * dist / tl, at(ga_pl, 5, v - 1) = tv.z * dist / tl;
    const D3 mid = scl3(unit3(add3(f, t)), R);
    at(xr_pl, 0, v - 1) = mid.x, at(xr_pl, 1, v - 1) = mid.y, at(xr_pl, 2, v - 1) = mid.z;
  }
  double s = 0.0;
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    s = s + tri_area(c0, xt[v - 1], xt[vp - 1]);
  }
  const double area = s * R * R;
  at(gp_pl, 0, 0) = area;
  at(gp_pl, 1, 0) = 1.0 / area;
  // gradient coefficients of the pole centre and its ring
  const double f = 0.5 * at(gp_pl, 1, 0);
  for (int d = 0; d < 3; ++d) {
    double sum = 0.0;
    for (int v = 2; v <= 6; ++v) {
      const int vp = (v == 6) ? 2 : v + 1;
      sum = sum + 2.0 * (at(gt_pl, 2, v - 1) - 1.0) * at(ga_pl, d, vp - 1);
    }
    cg_pl[((size_t)p * 3 + d) * kGallPl + 0] = sum * f;
    for (int v = 2; v <= 6; ++v) {
      const int vp = (v == 6) ? 2 : v + 1, vm = (v == 2) ? 6 : v - 1;
      cg_pl[((size_t)p * 3 + d) * kGallPl + v - 1] =
          (at(gt_pl, 4, vm - 1) * at(ga_pl, d, vm - 1) + at(gt_pl, 4, vm - 1) * at(ga_pl, d, v - 1) +
           at(gt_pl, 3, v - 1) * at(ga_pl, d, v - 1) + at(gt_pl, 3, v - 1) * at(ga_pl, d, vp - 1)) *
          f;
    }
  }
}

// corners (W, S, E, N) of the ten diamonds, as unit vectors: diamonds 1-5 have the north pole
// as corner N, 6-10 the south pole as corner S (the region table of mod_adm.f90:662-671)
static void diamond_corners(double out[10][4][3]) {
  const double lat = std::atan(0.5), pi = 3.14159265358979323846;
  double up[5][3], lo[5][3];
  for (int k = 0; k < 5; ++k) {
    const double a = 72.0 * k * pi / 180.0, b = (72.0 * k + 36.0) * pi / 180.0;
    up[k][0] = std::cos(lat) * std::cos(a), up[k][1] = std::cos(lat) * std::sin(a), up[k][2] = std::sin(lat);
    lo[k][0] = std::cos(lat) * std::cos(b), lo[k][1] = std::cos(lat) * std::sin(b), lo[k][2] = -std::sin(lat);
  }
  const double np[3] = {0.0, 0.0, 1.0}, sp[3] = {0.0, 0.0, -1.0};
  auto set = [&](int d, int c, const double *v) {
    for (int x = 0; x < 3; ++x) out[d][c][x] = v[x];
  };
  for (int k = 0; k < 5; ++k) set(k, 0, up[k]), set(k, 1, lo[k]), set(k, 2, up[(k + 1) % 5]), set(k, 3, np);
  for (int k = 0; k < 5; ++k) {
    const int d = (k == 0) ? 5 : 10 - k;
    set(d, 0, lo[(k + 4) % 5]), set(d, 1, sp), set(d, 2, lo[k]), set(d, 3, up[k]);
  }
}

}  // namespace icoadv

using namespace icoadv;

extern "C" int ica_grid_build_dev(ica_ctx *ctx, double radius, double *GRD_x, double *GRD_x_pl, double *GRD_xr,
                                  double *GRD_xr_pl, double *GMTR_p, double *GMTR_p_pl, double *GMTR_t,
                                  double *GMTR_t_pl, double *GMTR_a, double *GMTR_a_pl, double *coef_grad,
                                  double *coef_grad_pl) {
  if (!ctx) return set_error("ica_grid_build_dev: NULL context"), ICA_ERR_ARG;
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  int rc = c->need_grid("ica_grid_build_dev");
  if (rc) return rc;
  if (!GRD_x || !GRD_x_pl || !GRD_xr || !GRD_xr_pl || !GMTR_p || !GMTR_p_pl || !GMTR_t || !GMTR_t_pl || !GMTR_a ||
      !GMTR_a_pl || !coef_grad || !coef_grad_pl || !(radius > 0.0))
    return set_error("ica_grid_build_dev: bad argument"), ICA_ERR_ARG;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  const Topology &t = *c->topo;
  const int G = t.gall_1d, L = t.nrgn, n = 1 << t.glevel;
  const size_t gall = (size_t)G * G, plane = (size_t)L * gall, nlat = (size_t)10 * (n + 1) * (n + 1) * 3;
  double *lat = (double *)c->buf("geo_lattice", nlat * sizeof(double));
  double *xu = (double *)c->buf("geo_xu", 3 * plane * sizeof(double));
  double *xu_pl = (double *)c->buf("geo_xu_pl", 3 * kLallPl * kGallPl * sizeof(double));
  double *xt = (double *)c->buf("geo_xt", 6 * plane * sizeof(double));
  double *corners = (double *)c->buf("geo_corners", 120 * sizeof(double));
  if (!lat || !xu || !xu_pl || !xt || !corners) return set_error("ica_grid_build_dev: cudaMalloc"), ICA_ERR_NOMEM;
  double hc[10][4][3];
  diamond_corners(hc);
  cudaStream_t st = c->stream;
  e = cudaMemcpyAsync(corners, hc, sizeof(hc), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "ica_grid_build_dev: corners");
  e = cudaStreamSynchronize(st);  // hc is a stack array
  if (e != cudaSuccess) return cuda_fail(e, "ica_grid_build_dev: corners");
  long long launches = 0;
  auto blocks = [](long long work) { return (unsigned)((work + 255) / 256); };
  k_geo_lattice_corners<<<1, 32, 0, st>>>(lat, n, corners), ++launches;
  for (int h = n; h > 1; h /= 2) {
    const long long m = n / (h / 2) + 1;
    k_geo_lattice_level<<<blocks(10 * m * m), 256, 0, st>>>(lat, n, h), ++launches;
  }
  k_geo_positions<<<blocks((long long)plane), 256, 0, st>>>(lat, n, 1 << t.rlevel, t.nmax, G, L, xu, xu_pl),
      ++launches;
  const Plan &p = c->plan[0];
  launch_gather<double>(c->D, p.n, p.dst, p.src, 1, 3, xu, xu_pl, st), ++launches;  // halos of the positions
  k_geo_scale<<<blocks(3LL * plane), 256, 0, st>>>(xu, xu_pl, 3 * plane, radius, GRD_x, GRD_x_pl), ++launches;
  k_geo_tri<<<blocks((long long)plane), 256, 0, st>>>(xu, G, L, radius, xt, GMTR_t), ++launches;
  k_geo_tri_fix<<<(L + 63) / 64, 64, 0, st>>>(G, L, c->d_have_sgp, xt, GMTR_t), ++launches;
  k_geo_arc<<<blocks(3LL * plane), 256, 0, st>>>(xt, G, L, c->d_have_sgp, radius, GMTR_a, GRD_xr), ++launches;
  k_geo_area<<<blocks((long long)plane), 256, 0, st>>>(xu, xt, G, L, c->d_have_sgp, radius, GMTR_p), ++launches;
  k_geo_poles<<<1, 32, 0, st>>>(xu_pl, radius, GRD_xr_pl, GMTR_p_pl, GMTR_t_pl, GMTR_a_pl, coef_grad_pl),
      ++launches;
  // halo areas from the neighbour regions and the pole centres, as after a COMM of GMTR_p; the
  // pole arrays keep only their centre values (the fill runs on a copy of them)
  double *gp_pl_fill = (double *)c->buf("geo_gp_pl", 8 * kLallPl * kGallPl * sizeof(double));
  if (!gp_pl_fill) return set_error("ica_grid_build_dev: cudaMalloc"), ICA_ERR_NOMEM;
  e = cudaMemcpyAsync(gp_pl_fill, GMTR_p_pl, 8 * kLallPl * kGallPl * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "ica_grid_build_dev: GMTR_p_pl");
  launch_gather<double>(c->D, p.n, p.dst, p.src, 1, 8, GMTR_p, gp_pl_fill, st), ++launches;
  e = cudaMemsetAsync(coef_grad, 0, (size_t)L * 21 * gall * sizeof(double), st);
  if (e != cudaSuccess) return cuda_fail(e, "ica_grid_build_dev: coef_grad");
  k_geo_grad<<<blocks(3LL * plane), 256, 0, st>>>(GMTR_t, GMTR_a, GMTR_p, G, L, c->d_have_sgp, coef_grad),
      ++launches;
  c->launches += launches;
  return c->check_launch("ica_grid_build_dev");
}
