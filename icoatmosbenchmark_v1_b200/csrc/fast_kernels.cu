// Batched tracer step: FP32 flux-form remap / limiter arithmetic on interior
// faces, FP64 on region-seam faces, FP64 rhog / rhogq mass update.
//
// Per step, on the context stream:
//   k_fast_boundary  gradient and Thuburn outflow bounds Qout (FP64) of every
//                    region-boundary cell and both pole centres, into bbuf.  These
//                    are exactly the values the reference's two mid-step halo
//                    exchanges (grad q and Qout, mod_src_tracer.f90:371) would move
//                    into other regions' halos, so no exchange is needed; the seam
//                    and pole passes read them.  One thread per (cell, level): the
//                    face geometry once, then the tracers.
//   k_fast_seam      FP64 flux and limited value of every seam face (below), all tracers.
//   k_fast_pole      the two pole centres (horizontal + vertical), FP64.
//   k_fast_faces     per (owner cell, level): the flux of its three faces (FP32 triangle
//                    values; the seam pass's FP64 value on seams), the owner-side upwind
//                    mask and the remap displacement of each face's upwind cell.
//   k_fast_horiz     horizontal sub-step: one CTA per (region tile, 8 levels; one level per
//                    work item in the persistent form for batches of grids), one thread per
//                    cell of the tile and its 1-wide ring; the tracer-independent set-up of a
//                    level (Courant numbers, outflow faces, Thuburn sums), then per batch of
//                    TB tracers two phases with a barrier each: every ring cell's gradient,
//                    Qout, face bounds and the limited values of its outflow faces; then the
//                    FP64 update of the tile cells and q of the next batch from its TMA window.
//   k_fast_vert      vertical sub-step: one thread per (column, 4 tracers) streaming the
//                    levels through a 3-level shared-memory ring of its own cp.async copies,
//                    limiter two levels behind, FP64 update in place.
//   k_fast_carry     halo points that no halo list writes keep their input values.
//   gather           halo/pole fill of the new state (the COMM plan).
//
// Faces are "seam" faces when one of their two cells is a halo cell; the
// neighbouring region computes the same face from its own halo copy, so those
// faces are done in FP64 (k_fast_seam) from the FP64 boundary values.  An
// interior face is computed by every tile that needs it from the same inputs by the same
// instructions (cell positions enter only through the per-face offsets GRD_xr - GRD_x,
// fixed per face), so both of its cells see the same value and the flux form conserves
// mass to FP64 rounding.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "fast_common.cuh"
#include "fast_kernels.cuh"

namespace icoadv {

// ---- accessors on global memory (FP64 values at region coords of one (l,k) slab)
struct GFields {
  const FastInst *I;
  int l, k;
  __device__ double operator()(int var, int i, int j) const {
    const size_t off = ((size_t)l * I->K + k) * I->gall + (size_t)(j - 1) * I->G + (i - 1);
    if (var == 0) return I->rho_in[off];
    return fld(*I, var - 1, off);
  }
};
// ---- poles: the 5 ring faces of pole p at level k (mod_src_tracer.f90:326-374), FP64
__device__ void pole_faces(const FastInst &I, int p, int k, double flux[7], double xc[7][3]) {
  const size_t off = ((size_t)p * I.K + k) * kGallPl;
  auto GT = [&](int v, int w) { return I.GMTR_t_pl[((size_t)(w - 1) * kLallPl + p) * kGallPl + (v - 1)]; };
  auto GA = [&](int v, int h) { return I.GMTR_a_pl[((size_t)(h - 1) * kLallPl + p) * kGallPl + (v - 1)]; };
  auto R = [&](int v) { return I.rho_in_pl[off + v - 1]; };
  auto X = [&](int v) { return fld_pl(I, 0, off + v - 1); };
  auto Y = [&](int v) { return fld_pl(I, 1, off + v - 1); };
  auto Z = [&](int v) { return fld_pl(I, 2, off + v - 1); };
  double rt[7], xt[7], yt[7], zt[7];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1;
    rt[v] = R(1) * GT(v, W1) + R(v) * GT(v, W2) + R(vp) * GT(v, W3);
    xt[v] = X(1) * GT(v, W1) + X(v) * GT(v, W2) + X(vp) * GT(v, W3);
    yt[v] = Y(1) * GT(v, W1) + Y(v) * GT(v, W2) + Y(vp) * GT(v, W3);
    zt[v] = Z(1) * GT(v, W1) + Z(v) * GT(v, W2) + Z(vp) * GT(v, W3);
  }
  for (int v = 2; v <= 6; ++v) {
    const int vm = (v == 2) ? 6 : v - 1;
    const double rr = 1.0 / mx64(rt[vm] + rt[v], DBL_EPSILON);
    const double vx = xt[vm] + xt[v], vy = yt[vm] + yt[v], vz = zt[vm] + zt[v];
    flux[v] = 0.5 * (vx * GA(v, HNX) + vy * GA(v, HNY) + vz * GA(v, HNZ));
    for (int x = 0; x < 3; ++x) {
      const double xr = I.GRD_xr_pl[((size_t)x * kLallPl + p) * kGallPl + (v - 1)];
      xc[v][x] = xr - (x == 0 ? vx : (x == 1 ? vy : vz)) * rr * I.dt * 0.5;
    }
  }
}

// Qout of pole centre p at level k (mod_src_tracer.f90:307-363), d = 0, from q at its 6 points
__device__ void pole_qout(const FastInst &I, int p, int k, const double q[7], const double flux[7], double &Qmin,
                          double &Qmax) {
  const size_t off = ((size_t)p * I.K + k) * kGallPl;
  const double rarea = I.GMTR_p_pl[((size_t)(P_RAREA - 1) * kLallPl + p) * kGallPl];
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  double qmin1[7], qmax1[7], chm[7], ch[7];
  for (int v = 2; v <= 6; ++v) {
    const int vp = (v == 6) ? 2 : v + 1, vm = (v == 2) ? 6 : v - 1;
    const double lo = mn64(mn64(mn64(q[1], q[v]), q[vm]), q[vp]);
    const double hi = mx64(mx64(mx64(q[1], q[v]), q[vm]), q[vp]);
    ch[v] = flux[v] * rarea * I.dt / I.rho_in_pl[off];
    const double c = 0.5 - fsg(0.5, ch[v] - EPS);
    qmin1[v] = c * lo + (1.0 - c) * BIG;
    qmax1[v] = c * hi + (1.0 - c) * (-BIG);
    chm[v] = c * ch[v];
  }
  double qnmin = q[1], qnmax = q[1];
  for (int v = 2; v <= 6; ++v) qnmin = mn64(qnmin, qmin1[v]), qnmax = mx64(qnmax, qmax1[v]);
  double Cin = 0, Cout = 0, CQmax = 0, CQmin = 0;
  for (int v = 2; v <= 6; ++v) {
    Cin = Cin + chm[v];
    Cout = Cout - chm[v] + ch[v];
    CQmin = CQmin + chm[v] * qmin1[v];
    CQmax = CQmax + chm[v] * qmax1[v];
  }
  const double zerosw = 0.5 - fsg(0.5, fabs(Cout) - EPS);
  const double qn = q[1];
  Qmin = (qn - CQmax - qnmax * (1.0 - Cin - Cout + 0.0)) / (Cout + zerosw) * (1.0 - zerosw) + qn * zerosw;
  Qmax = (qn - CQmin - qnmin * (1.0 - Cin - Cout + 0.0)) / (Cout + zerosw) * (1.0 - zerosw) + qn * zerosw;
}

// ---- boundary pass: FP64 gradient and Qout (mod_src_tracer.f90:143-282, d = 0) of the
// region-boundary cells and the pole centres, one thread per (entry, level), all tracers.
__global__ void k_fast_boundary(const __grid_constant__ MultiInst M) {
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = find_inst(M, tid, [](const FastInst &J) { return (long long)J.nb * (J.K - 2); });
  if (ii < 0) return;
  const FastInst &I = M.inst[ii];
  const int b = (int)(tid % I.nb);
  const int k = 1 + (int)(tid / I.nb);
  const int p = I.blist[b];
  if (!owns_point(I, p)) return;  // another rank's boundary cell or pole centre
  const size_t tstride = (size_t)I.lall * I.K * I.gall;
  double *dst0 = I.bbuf + ((size_t)k * I.nb + b) * 5;
  const size_t dstride = (size_t)I.K * I.nb * 5;  // next tracer
  if (p >= I.lall * I.gall) {  // pole centre
    const int pl = (p - I.lall * I.gall) / kGallPl;
    const size_t off = ((size_t)pl * I.K + k) * kGallPl;
    const size_t tsp = (size_t)kLallPl * I.K * kGallPl;
    double flux[7], xc[7][3], rinv[7];
    pole_faces(I, pl, k, flux, xc);
    for (int v = 1; v <= 6; ++v) rinv[v] = 1.0 / I.rho_in_pl[off + v - 1];
    for (int t = 0; t < I.ntr; ++t) {
      double q[7], out[5];
      for (int v = 1; v <= 6; ++v) q[v] = I.Q_in_pl[t * tsp + off + v - 1] * rinv[v];
      for (int x = 0; x < 3; ++x) {
        const double *cx = I.cg_pl + ((size_t)pl * 3 + x) * 6;
        double s = cx[0] * q[1];
        for (int v = 2; v <= 6; ++v) s = s + cx[v - 1] * q[v];
        out[x] = s;
      }
      pole_qout(I, pl, k, q, flux, out[3], out[4]);
      double *dst = dst0 + t * dstride;
      for (int x = 0; x < 5; ++x) dst[x] = out[x];
    }
    return;
  }
  const int l = p / I.gall, c = p % I.gall;
  const int G = I.G, i = c % G + 1, j = c / G + 1;
  const bool sgp = I.have_sgp[l] != 0;
  const GFields f{&I, l, k};
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  // tracer-independent: Courant numbers and upwind masks of the 6 faces, 1/rho on the 3x3 block
  const int oi[7] = {0, i, i, i, i - 1, i - 1, i}, oj[7] = {0, j, j, j, j, j - 1, j - 1};
  const int fa[7] = {0, AI, AIJ, AJ, AI, AIJ, AJ};
  const double rho_c = f(0, i, j), ra_c = rarea(I, l, i, j);
  double ch[7], chm[7], cmk[7];
  for (int m = 1; m <= 6; ++m) {
    double xcv[3];
    const bool ex = face_exists(I, oi[m], oj[m], fa[m]);
    const double fl = ex ? face_geo(I, l, oi[m], oj[m], fa[m], sgp, f, xcv) : 0.0;
    const double flx = ex ? cell_flx(I, l, i, j, m, sgp, fl, ra_c) : 0.0;
    ch[m] = flx / rho_c;
    chm[m] = mn64(ch[m], 0.0);
    const double ch_own = (m <= 3) ? ch[m] : (fl * rarea(I, l, oi[m], oj[m]) * I.dt) / f(0, oi[m], oj[m]);
    cmk[m] = 0.5 - fsg(0.5, ch_own - EPS);
  }
  const double Cin = chm[1] + chm[2] + chm[3] + chm[4] + chm[5] + chm[6];
  const double Cout =
      ch[1] - chm[1] + ch[2] - chm[2] + ch[3] - chm[3] + ch[4] - chm[4] + ch[5] - chm[5] + ch[6] - chm[6];
  const double zerosw = 0.5 - fsg(0.5, fabs(Cout) - EPS);
  const double rden = (1.0 - zerosw) / (Cout + zerosw), omc = 1.0 - Cin - Cout;
  double rinv[3][3];
  for (int dj = 0; dj < 3; ++dj)
    for (int di = 0; di < 3; ++di) rinv[dj][di] = 1.0 / f(0, i - 1 + di, j - 1 + dj);
  double cgr[3][7];
  for (int x = 0; x < 3; ++x)
    for (int n = 0; n < 7; ++n) cgr[x][n] = I.cg[(((size_t)l * 3 + x) * 7 + n) * I.gall + c];
  const int di7[7] = {0, 1, 1, 0, -1, -1, 0}, dj7[7] = {0, 0, 1, 1, 0, -1, -1};
  // The 4 points of each face's bounds (bounds64 for the face's owner), as offsets in the 3x3
  // block: a region-boundary cell lies in [gmin, gmax]^2, so every point is in the block and
  // no index clamp applies.  Face 5's owner is the singular corner (gmin-1, gmin-1) when the
  // cell is (gmin, gmin) of a region with the singular point: then its points shift.
  const bool sgp5 = sgp && i == I.gmin && j == I.gmin;
  // rhogq of the 3x3 block, one tracer ahead: the next tracer's loads are issued before this
  // tracer's stores (which the compiler may not move them across)
  const double *Q0 = I.Q_in + ((size_t)l * I.K + k) * I.gall + (size_t)(j - 2) * G + (i - 2);
  double raw[3][3];
#pragma unroll
  for (int dj = 0; dj < 3; ++dj)
#pragma unroll
    for (int di = 0; di < 3; ++di) raw[dj][di] = Q0[(size_t)dj * G + di];
  for (int t = 0; t < I.ntr; ++t) {
    double q9[3][3];
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
      for (int di = 0; di < 3; ++di) q9[dj][di] = raw[dj][di] * rinv[dj][di];
    if (t + 1 < I.ntr) {
      const double *Qn = Q0 + (size_t)(t + 1) * tstride;
#pragma unroll
      for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) raw[dj][di] = Qn[(size_t)dj * G + di];
    }
    auto Q = [&](int di, int dj) { return q9[dj + 1][di + 1]; };
    double out[5];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      double s = cgr[x][0] * q9[1][1];
#pragma unroll
      for (int n = 1; n <= 6; ++n) s = s + cgr[x][n] * q9[1 + dj7[n]][1 + di7[n]];
      out[x] = s;
    }
    // (q0, b, c, d) of bounds64, in its order
    double lo[7], hi[7];
    auto b4 = [&](int m, double q0, double b, double c, double d) {
      lo[m] = mn64(mn64(mn64(q0, b), c), d);
      hi[m] = mx64(mx64(mx64(q0, b), c), d);
    };
    b4(1, Q(0, 0), Q(0, -1), Q(1, 0), Q(1, 1));     // AI of (i, j)
    b4(2, Q(0, 0), Q(1, 0), Q(1, 1), Q(0, 1));      // AIJ of (i, j)
    b4(3, Q(0, 0), Q(1, 1), Q(0, 1), Q(-1, 0));     // AJ of (i, j)
    b4(4, Q(-1, 0), Q(-1, -1), Q(0, 0), Q(0, 1));   // AI of (i-1, j)
    if (sgp5) b4(5, Q(-1, -1), Q(0, 0), Q(1, 0), Q(-1, 0));  // AIJ of the singular corner
    else b4(5, Q(-1, -1), Q(0, -1), Q(0, 0), Q(-1, 0));      // AIJ of (i-1, j-1)
    b4(6, Q(0, -1), Q(1, 0), Q(0, 0), Q(-1, -1));   // AJ of (i, j-1)
    double qmn[7], qmx[7];
#pragma unroll
    for (int m = 1; m <= 6; ++m) {
      const double cm = cmk[m];
      if (m <= 3) qmn[m] = cm * lo[m] + (1.0 - cm) * BIG, qmx[m] = cm * hi[m] + (1.0 - cm) * (-BIG);
      else qmn[m] = cm * BIG + (1.0 - cm) * lo[m], qmx[m] = cm * (-BIG) + (1.0 - cm) * hi[m];
    }
    const double q0 = q9[1][1];
    double qnmin = q0, qnmax = q0;
#pragma unroll
    for (int m = 1; m <= 6; ++m) qnmin = mn64(qnmin, qmn[m]);
#pragma unroll
    for (int m = 1; m <= 6; ++m) qnmax = mx64(qnmax, qmx[m]);
    const double CQmin = chm[1] * qmn[1] + chm[2] * qmn[2] + chm[3] * qmn[3] + chm[4] * qmn[4] + chm[5] * qmn[5] +
                         chm[6] * qmn[6];
    const double CQmax = chm[1] * qmx[1] + chm[2] * qmx[2] + chm[3] * qmx[3] + chm[4] * qmx[4] + chm[5] * qmx[5] +
                         chm[6] * qmx[6];
    out[3] = (q0 - CQmax - qnmax * omc) * rden + q0 * zerosw;
    out[4] = (q0 - CQmin - qnmin * omc) * rden + q0 * zerosw;
    double *dst = dst0 + t * dstride;
#pragma unroll
    for (int x = 0; x < 5; ++x) dst[x] = out[x];
  }
}

__device__ __forceinline__ const double *bval(const FastInst &I, int t, int k, int b) {
  return I.bbuf + (((size_t)t * I.K + k) * I.nb + b) * 5;
}

// ---- seam faces (one side a halo cell): FP64 flux once per (face, level), then the limited
// value of every tracer.  The face's Courant number and upwind mask, the remap offsets and
// 1/rho of the cells involved do not depend on the tracer and are formed once.
__global__ void k_fast_seam(const __grid_constant__ MultiInst M) {
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = find_inst(M, tid, [](const FastInst &J) { return (long long)J.ns * (J.K - 2); });
  if (ii < 0) return;
  const FastInst &I = M.inst[ii];
  const int sidx = (int)(tid % I.ns), k = 1 + (int)(tid / I.ns);
  const int code = I.seam_list[sidx];
  const int a = code % 3 + 1, p = code / 3;
  if (!owns_point(I, p)) return;  // a face of another rank's region
  const int l = p / I.gall, c = p % I.gall;
  const int G = I.G, i = c % G + 1, j = c / G + 1;
  const bool sgp = I.have_sgp[l] != 0;
  const GFields gf{&I, l, k};
  double xc[3];
  const double fl = face_geo(I, l, i, j, a, sgp, gf, xc);
  I.sflux[(size_t)k * I.ns + sidx] = fl;
  const int ni = (a == AI || a == AIJ) ? i + 1 : i, nj = (a == AIJ || a == AJ) ? j + 1 : j;
  const double ch = (fl * rarea(I, l, i, j) * I.dt) / gf(0, i, j);
  const double cm = 0.5 - fsg(0.5, ch - DBL_EPSILON);
  const int bo = I.bsrc[(size_t)l * I.gall + (j - 1) * G + (i - 1)];
  const int bn = I.bsrc[(size_t)l * I.gall + (nj - 1) * G + (ni - 1)];
  double dxo[3], dxn[3];
  for (int x = 0; x < 3; ++x) dxo[x] = xc[x] - gx(I, l, i, j, x), dxn[x] = xc[x] - gx(I, l, ni, nj, x);
  // the 4 cells of the face's bounds (bounds64's selection) and 1/rho there; the owner is [0]
  int pc[4];
  {
    const int ij = (j - 1) * G + i;
    int im1j = ij - 1, ijm1 = ij - G;
    if (im1j < 1) im1j = 1;
    if (ijm1 < 1) ijm1 = 1;
    pc[0] = ij;
    if (a == AI) pc[1] = ijm1, pc[2] = ij + 1, pc[3] = ij + G + 1;
    else if (a == AIJ) {
      if (sgp && i == I.gmin - 1 && j == I.gmin - 1) pc[1] = ij + G + 1, pc[2] = ij + G + 2, pc[3] = ij + G;
      else pc[1] = ij + 1, pc[2] = ij + G + 1, pc[3] = ij + G;
    } else pc[1] = ij + G + 1, pc[2] = ij + G, pc[3] = im1j;
  }
  const size_t slab = ((size_t)l * I.K + k) * I.gall, tstride = (size_t)I.lall * I.K * I.gall;
  const size_t on = (size_t)(nj - 1) * G + (ni - 1);
  double rv[4];
  for (int n = 0; n < 4; ++n) rv[n] = 1.0 / I.rho_in[slab + pc[n] - 1];
  const double rn = 1.0 / I.rho_in[slab + on];
  const double BIG = DBL_MAX;
  // the tracer's inputs one tracer ahead: the next tracer's loads are issued before this
  // tracer's store (which the compiler may not move them across).  Per-tracer strides are
  // applied to base pointers (the index products stay out of the tracer loop).
  double rq[5], rgo[5], rgn[5];
  const double *Qt = I.Q_in + slab;
  const size_t bstride = (size_t)I.K * I.nb * 5, vstride = (size_t)I.K * I.ns;
  const double *bvo = I.bbuf + ((size_t)k * I.nb + (bo >= 0 ? bo : 0)) * 5;
  const double *bvn = I.bbuf + ((size_t)k * I.nb + (bn >= 0 ? bn : 0)) * 5;
  auto fetch = [&]() {
#pragma unroll
    for (int n = 0; n < 4; ++n) rq[n] = Qt[pc[n] - 1];
    rq[4] = Qt[on];
#pragma unroll
    for (int x = 0; x < 5; ++x) rgo[x] = bo >= 0 ? bvo[x] : 0.0, rgn[x] = bn >= 0 ? bvn[x] : 0.0;
    Qt += tstride, bvo += bstride, bvn += bstride;
  };
  fetch();
  const size_t vbase = (size_t)k * I.ns + sidx;
  float *sv32 = I.f64 ? nullptr : I.sval + vbase;
  double *sv64 = I.f64 ? I.sval64 + vbase : nullptr;
  for (int t = 0; t < I.ntr; ++t) {
    double qv[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) qv[n] = rq[n] * rv[n];
    const double qo = qv[0], qn = rq[4] * rn;
    // gradient and Qout of both cells (boundary or halo cells of this region)
    double go[5] = {0, 0, 0, 0, 0}, gn[5] = {0, 0, 0, 0, 0};
    if (bo >= 0) for (int x = 0; x < 5; ++x) go[x] = rgo[x];
    else go[3] = go[4] = qo;  // halo point no list reaches: Qout = q, grad = 0 (as after the reference fill)
    if (bn >= 0) for (int x = 0; x < 5; ++x) gn[x] = rgn[x];
    else gn[3] = gn[4] = qn;
    if (t + 1 < I.ntr) fetch();
    double vu = qn, vs = qo;
    for (int x = 0; x < 3; ++x) vu = vu + gn[x] * dxn[x];
    for (int x = 0; x < 3; ++x) vs = vs + go[x] * dxo[x];
    double v = cm * vu + (1.0 - cm) * vs;
    const double lo = mn64(mn64(mn64(qv[0], qv[1]), qv[2]), qv[3]);
    const double hi = mx64(mx64(mx64(qv[0], qv[1]), qv[2]), qv[3]);
    const double own_min = cm * lo + (1.0 - cm) * BIG, own_max = cm * hi + (1.0 - cm) * (-BIG);
    const double nb_min = cm * BIG + (1.0 - cm) * lo, nb_max = cm * (-BIG) + (1.0 - cm) * hi;
    v = cm * mn64(mx64(v, own_min), own_max) + (1.0 - cm) * mn64(mx64(v, nb_min), nb_max);
    v = cm * mx64(mn64(v, gn[4]), gn[3]) + (1.0 - cm) * mx64(mn64(v, go[4]), go[3]);
    if (I.f64) *sv64 = v, sv64 += vstride;
    else *sv32 = (float)v, sv32 += vstride;
  }
}

// ---- per-face remap offsets GRD_xr - GRD_x of the owner and of the neighbour (FP32),
// fixed per face, so an interior face value does not depend on the tile that computes it.
// off32 (lall, 18, gall): [a*6 + x] owner side, [a*6 + 3 + x] neighbour side, a = face 0..2.
// After them the face geometry k_fast_faces reads, in the arithmetic type (lall, 16, gall):
// TI W1..W3, TJ W1..W3 (GMTR_t), HNX..HNZ of faces AI, AIJ, AJ (GMTR_a), rarea (GMTR_p).
template <typename T>
__global__ void k_fast_offsets(FastInst I, T *off) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)I.lall * I.gall) return;
  const int l = (int)(tid / I.gall), c = (int)(tid % I.gall);
  const int G = I.G, i = c % G + 1, j = c / G + 1;
  for (int a = 1; a <= 3; ++a) {
    const int ni = (a == AI || a == AIJ) ? i + 1 : i, nj = (a == AIJ || a == AJ) ? j + 1 : j;
    const bool nok = ni <= G && nj <= G;
    for (int x = 0; x < 3; ++x) {
      const double xr = gxr(I, l, i, j, a, x + 1);
      off[((size_t)l * kOffPlanes + (a - 1) * 6 + x) * I.gall + c] = (T)(xr - gx(I, l, i, j, x));
      off[((size_t)l * kOffPlanes + (a - 1) * 6 + 3 + x) * I.gall + c] = nok ? (T)(xr - gx(I, l, ni, nj, x)) : T(0);
    }
  }
  T *geo = off + (size_t)I.lall * kOffPlanes * I.gall + (size_t)l * kFaceGeoPlanes * I.gall + c;
  for (int w = 0; w < 3; ++w) {
    geo[(size_t)w * I.gall] = (T)gt(I, l, i, j, TI, W1 + w);
    geo[(size_t)(3 + w) * I.gall] = (T)gt(I, l, i, j, TJ, W1 + w);
  }
  for (int a = 0; a < 3; ++a)
    for (int h = 0; h < 3; ++h) geo[(size_t)(6 + 3 * a + h) * I.gall] = (T)ga(I, l, i, j, a + 1, HNX + h);
  geo[(size_t)15 * I.gall] = (T)rarea(I, l, i, j);
}

// Threshold of the upwind masks (0.5 - sign(0.5, ch - EPS)) and of the zero-outflow guards
// (zerosw) in either arithmetic: the FP64 EPS, also in FP32, not epsilon(1.0).  These are switches, not
// roundings: with FP32's own EPS a face whose Courant number lies in (2.2e-16, 1.2e-7) is
// taken from the other side than in FP64, which moves its 4-point bounds into or out of the
// cell's qnext; at a slotted-cylinder edge (glevel 7, kall 96) that gave 9e-4 relative error
// against the FP64 oracle in 10 cells.  With the FP64 threshold the same run is at 1.6e-7.
// (The standalone *_f32 kernel entry points keep the reference's RP = SP semantics.)
template <typename R>
__device__ __forceinline__ R eps_thr() { return (R)DBL_EPSILON; }

// Face fluxes of every owner cell and level, once per step (dyn_horiz_adv_flux/src/
// mod_src_tracer.f90:141-309): FP32 triangle values and faces between interior cells, the
// FP64 value of k_fast_seam on seam faces, zero where the reference has no face.  With each
// face the owner-side upwind mask (cmask of horizontal_limiter_thuburn, from the owner's
// Courant number) and the remap displacement of the upwind cell: GRD_xc - GRD_x of that
// cell, i.e. the fixed per-face offset GRD_xr - GRD_x of its side plus the centroid
// displacement -rhov rr dt / 2.  One thread per (owner cell, level); every tile that needs a
// face reads these values, so the face's two cells see the same flux and mask.
template <typename R>
__global__ void k_fast_faces(const __grid_constant__ MultiInst M) {
  using A = Arith<R>;
  long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = find_inst(M, w, [](const FastInst &I) { return (long long)(I.l1 - I.l0) * (I.K - 2) * I.gall; });
  if (ii < 0) return;
  const FastInst &I = M.inst[ii];
  // 32-bit index arithmetic throughout (a 64-bit division or product is several times the
  // cost of this thread's arithmetic); the host keeps 3 * lall * kall * gall below 2^31
  const unsigned wu = (unsigned)w, gall = (unsigned)I.gall, kin = (unsigned)(I.K - 2), Gu = (unsigned)I.G;
  const int G = I.G, c = (int)(wu % gall);
  const unsigned lk = wu / gall;
  const int k = 1 + (int)(lk % kin), l = I.l0 + (int)(lk / kin);
  const int i = (int)((unsigned)c % Gu) + 1, j = (int)((unsigned)c / Gu) + 1;
  const unsigned n3 = (unsigned)I.lall * (unsigned)I.K * gall, o = ((unsigned)l * (unsigned)I.K + (unsigned)k) * gall + c;
  const R dtf = (R)I.dt;
  auto interior = [&](int a, int b) { return a >= I.gmin && a <= I.gmax && b >= I.gmin && b <= I.gmax; };
  // faces between interior cells take the FP32 triangle form, seam faces the FP64 value of
  // k_fast_seam; AI = TJ(i,j-1) + TI(i,j), AIJ = TI(i,j) + TJ(i,j), AJ = TJ(i,j) + TI(i-1,j),
  // so the four triangles are formed once each, before any store
  bool ex[3], inner[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int ni = (a < 2) ? i + 1 : i, nj = (a > 0) ? j + 1 : j;
    ex[a] = i < G && j < G && face_exists(I, i, j, a + 1);
    inner[a] = ex[a] && interior(i, j) && interior(ni, nj);
  }
  // the per-column face geometry of this region (see k_fast_offsets) and the fields of the six
  // cells the four triangles touch: (i,j), (i+1,j), (i+1,j+1), (i,j+1), (i,j-1), (i-1,j); an
  // inner face has all six inside the region's array
  const R *geo = fast_face_geo(sizeof(R) == 8 ? (const R *)(const void *)I.off64 : (const R *)(const void *)I.off32, I) +
                 (unsigned)l * kFaceGeoPlanes * gall + c;
  auto cellf = [&](int off, R f[4]) {
    const unsigned q = (unsigned)((int)o + off);
    f[0] = (R)I.rho_in[q];
    if (sizeof(R) == 8) f[1] = (R)I.vx64[q], f[2] = (R)I.vy64[q], f[3] = (R)I.vz64[q];
    else f[1] = (R)I.vx[q], f[2] = (R)I.vy[q], f[3] = (R)I.vz[q];
  };
  // triangle value v = f0 w1 + f1 w2 + f2 w3 with the weights at geometry offset gofs
  auto tri = [&](const R f0[4], const R f1[4], const R f2[4], int gofs, int wp, R v[4]) {
    const R w1 = geo[(int)wp * (int)gall + gofs], w2 = geo[(int)(wp + 1) * (int)gall + gofs],
            w3 = geo[(int)(wp + 2) * (int)gall + gofs];
#pragma unroll
    for (int x = 0; x < 4; ++x) v[x] = f0[x] * w1 + f1[x] * w2 + f2[x] * w3;
  };
  R tIij[4] = {}, tJij[4] = {}, tJm[4] = {}, tIm[4] = {};
  if (inner[0] || inner[1] || inner[2]) {
    R f00[4], f10[4], f11[4], f01[4], f0m[4], fm0[4];
    cellf(0, f00), cellf(1, f10), cellf(G + 1, f11), cellf(G, f01);
    if (inner[0]) cellf(-G, f0m);
    if (inner[2]) cellf(-1, fm0);
    if (inner[0] || inner[1]) tri(f00, f10, f11, 0, 0, tIij);   // TI(i,j)
    if (inner[1] || inner[2]) tri(f00, f11, f01, 0, 3, tJij);   // TJ(i,j)
    if (inner[0]) tri(f0m, f10, f00, -G, 3, tJm);               // TJ(i,j-1)
    if (inner[2]) tri(fm0, f00, f01, -1, 0, tIm);               // TI(i-1,j)
  }
  double F[3];
  R d[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    F[a] = 0.0;
    d[a][0] = d[a][1] = d[a][2] = R(0.0);
    if (inner[a]) {
      const R *p = (a == 0) ? tJm : (a == 1 ? tIij : tJij);
      const R *q = (a == 0) ? tIij : (a == 1 ? tJij : tIm);
      const R vx = p[1] + q[1], vy = p[2] + q[2], vz = p[3] + q[3];
      const R rr = R(1.0) / A::mx(p[0] + q[0], A::RR_EPS);
      const R Ff = R(0.5) * (vx * geo[(6 + 3 * a) * gall] + vy * geo[(7 + 3 * a) * gall] + vz * geo[(8 + 3 * a) * gall]);
      F[a] = (double)Ff;
      d[a][0] = -(vx * rr * dtf * R(0.5));
      d[a][1] = -(vy * rr * dtf * R(0.5));
      d[a][2] = -(vz * rr * dtf * R(0.5));
    } else if (ex[a]) {  // seam face
      const int sid = I.seam_id[((unsigned)l * gall + c) * 3 + a];
      F[a] = I.sflux[(unsigned)k * (unsigned)I.ns + sid];
    }
  }
  // the owner's Courant number of each face and its upwind mask, in the form the tile kernel
  // used to form them (FP32 flux, rarea and 1/rho of the owner), and the upwind side's offset
  const R ra = geo[15 * gall], rinv = (R)(1.0 / I.rho_in[o]);
  const R EPSf = eps_thr<R>();
  const R *offs = (sizeof(R) == 8 ? (const R *)(const void *)I.off64 : (const R *)(const void *)I.off32) +
                  (unsigned)l * kOffPlanes * gall + c;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    I.Fg[a * n3 + o] = F[a];
    const R chown = ((R)F[a] * ra * dtf) * rinv;
    const bool cm = (R(0.5) - A::sgn(R(0.5), chown - EPSf)) != R(0.0);
    R v[3] = {R(0.0), R(0.0), R(0.0)};
    if (inner[a]) {
      const R *ob = offs + (a * 6 + (cm ? 3 : 0)) * gall;
#pragma unroll
      for (int x = 0; x < 3; ++x) v[x] = ob[x * gall] + d[a][x];
    }
    const R wm = cm ? R(1.0) : R(0.0);
    if (sizeof(R) == 8) I.dupc64[a * n3 + o] = make_double4(v[0], v[1], v[2], wm);
    else I.dupc[a * n3 + o] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)wm);
  }
}


// ---- vertical Thuburn limiter (dyn_vert_adv_limiter/src/mod_src_tracer.f90:107-186), d = 0, FP32:
// the tracer-independent part of a level (upwind flags, Courant sums) and the per-tracer bounds
template <typename R>
struct VLim {
  R infl, a1, a2, bl, bu, icm, rden, zsw;
};
template <typename R>
__device__ __forceinline__ VLim<R> vlim_params(R c1, R c2, R c1p) {
  using A = Arith<R>;
  VLim<R> v;
  v.infl = R(0.5) - A::sgn(R(0.5), c1);
  const R infu = R(0.5) + A::sgn(R(0.5), c1p);
  v.bl = (R(1.0) - v.infl) * A::BIG;
  v.bu = (R(1.0) - infu) * A::BIG;
  v.a1 = v.infl * c1;
  v.a2 = infu * c2;
  const R Cin = v.a1 + v.a2;
  const R Cout = (R(1.0) - v.infl) * c1 + (R(1.0) - infu) * c2;
  v.icm = Cin + Cout;
  v.zsw = R(0.5) - A::sgn(R(0.5), fabs(Cout) - eps_thr<R>());
  v.rden = (R(1.0) - v.zsw) / (Cout + v.zsw);
  return v;
}
template <typename R>
__device__ __forceinline__ void vlim_qout(const VLim<R> &v, R qm, R qk, R qp, R &Qmin, R &Qmax) {
  using A = Arith<R>;
  const R minL = A::mn(qk, qm) + v.bl, minU = A::mn(qk, qp) + v.bu;
  const R maxL = A::mx(qk, qm) - v.bl, maxU = A::mx(qk, qp) - v.bu;
  const R qnmin = A::mn(A::mn(minL, minU), qk), qnmax = A::mx(A::mx(maxL, maxU), qk);
  const R CQmin = v.a1 * minL + v.a2 * minU, CQmax = v.a1 * maxL + v.a2 * maxU;
  Qmin = ((qk - qnmax) + qnmax * v.icm - CQmax) * v.rden + qk * v.zsw;
  Qmax = ((qk - qnmin) + qnmin * v.icm - CQmin) * v.rden + qk * v.zsw;
}

// ---- horizontal sub-step -----------------------------------------------------------
// One CTA per (region tile, level), all tracers in batches of TB.  Local frame: cell (i,j)
// of the region -> (x,y) = (i - i0, j - j0); the tile is x in [0,TX), y in [0,TY); the ring
// (one thread per cell) x in [-1,TX], y in [-1,TY]; the window of rhogq and rhog that the
// ring's stencils read, x in [-3,TX+2], y in [-2,TY+1].  The window's first column i0-4 is
// even for even TX (i0 = gmin + TX*n), so a TMA copy of its FP64 rows starts on a 16-byte
// boundary, as the tensor copy requires.
template <int TX, int TY>
struct TileGeo {
  static_assert(TX % 2 == 0, "the window's first column must be even");
  static constexpr int RW = TX + 2, RH = TY + 2, NR = RW * RH;  // ring cells
  static constexpr int NT = (NR + 31) / 32 * 32;                // threads (whole warps)
  static constexpr int WW = TX + 6, WH = TY + 4, NW = WW * WH;  // window
};

template <int TX, int TY, int TB, typename R>
struct TileSmem {
  using V2 = typename Arith<R>::V2;
  using V4 = typename Arith<R>::V4;
  static constexpr int NT = TileGeo<TX, TY>::NT, NW = TileGeo<TX, TY>::NW;
  alignas(128) double stage[2][TB][NW];  // rhogq of the window, FP64, [tracer][y][x]: two batches in flight
  alignas(128) double rho[NW];           // rhog of the window
  double rinv[NW];                       // 1 / rhog (0 outside the array)
  // tracer pairs (x: tracer 2p, y: tracer 2p+1): one 8-byte access serves both, and a
  // half-warp (one ring row) touches consecutive slots, so no padding is needed for banks
  V2 q2[TB / 2][NW];
  V2 qa[TB / 2][3][NT];  // limited values of the faces owned by ring cells
  V4 dup[3][NT];         // owner faces: upwind cell's remap displacement, owner-side mask (k_fast_faces)
  double flx[6][NT];     // flx_h (FP64) of the 6 faces of a tile cell
  unsigned long long mbar[2];  // one per stage buffer: its TMA copies have landed
};

// ---- TMA and mbarrier helpers (this GPU's memory only; no cluster multicast)
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase of parity `parity` of barrier b, for 2 s at most (false: gave up).
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try(b, parity))
    if (global_ns() - t0 > 2000000000ull) return false;
  return true;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *m, int c0, int c1, int c2,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"((unsigned long long)m), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"((unsigned long long)m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
// one element global -> shared without a register (cp.async; 4 or 8 bytes, naturally aligned)
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async copies 4, 8 or 16 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(dst)), "l"(src), "n"((int)sizeof(T))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int TX, int TY, int TB, typename R>
__device__ __forceinline__ void tile_smem_init(TileSmem<TX, TY, TB, R> &s) {
  if (threadIdx.x == 0) {
    mbar_init(&s.mbar[0], 1);
    mbar_init(&s.mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
}

// Does the tile with first cell (i0, j0) need the region-edge code?  An interior tile's ring
// lies strictly inside [gmin, gmax]^2: every ring cell and its neighbours are interior cells,
// no face of the tile is a seam face or absent, and the singular corner is not in it.
template <int TX, int TY>
__device__ __forceinline__ bool edge_tile(const FastInst &I, int i0, int j0) {
  return !(i0 - 1 > I.gmin && i0 + TX < I.gmax && j0 - 1 > I.gmin && j0 + TY < I.gmax);
}

// one work item (tile, level) of instance I; `phase` holds the parity each stage barrier waits
// for next (bit b: barrier b).  Returns false if a wait for a TMA copy gave up (the error word
// is set; the caller stops).  I is taken by value and the body inlined once per call site, so
// every field of I stays a constant-bank operand.  EDGE = false is the interior-tile form
// (edge_tile false): the checks and the seam, absent-face and singular-corner paths compile away.
template <int TX, int TY, int TB, typename R, bool EDGE, bool BWO = false>
__device__ __forceinline__ bool horiz_item(const FastInst I, const TileMaps *T, const int tile, const int k,
                                           TileSmem<TX, TY, TB, R> &s, unsigned &phase, R (&cgr)[21],
                                           const bool load_cg = true, const bool pre = false,
                                           const int knext = -1) {
  using A = Arith<R>;
  using V2 = typename A::V2;
  using V4 = typename A::V4;
  using Gm = TileGeo<TX, TY>;
  constexpr int RW = Gm::RW, NR = Gm::NR, NT = Gm::NT, WW = Gm::WW, NW = Gm::NW;
  constexpr int TP = TB / 2;  // tracer pairs of a batch: one V2 holds tracers 2p and 2p+1
  constexpr int NSLOT = (NW + NT - 1) / NT;
  constexpr unsigned QBYTES = (unsigned)(TB * NW * sizeof(double)), RBYTES = (unsigned)(NW * sizeof(double));
  const int tiles_per_rgn = I.ntx * I.nty;
  const int l = tile / tiles_per_rgn;
  const int tr = tile % tiles_per_rgn;
  const int i0 = I.gmin + (tr % I.ntx) * TX, j0 = I.gmin + (tr / I.ntx) * TY;
  const int tid = threadIdx.x;
  const int G = I.G, K = I.K, ntr = I.ntr;
  const int nbat = (ntr + TB - 1) / TB;
  const bool sgp = I.have_sgp[l] != 0;
  const size_t slab = (size_t)I.gall, n3 = (size_t)I.lall * K * I.gall;
  const size_t base = ((size_t)l * K + k) * slab;
  const double dt = I.dt;
  const R dtf = (R)dt;
  const R BIGf = A::BIG, EPSf = eps_thr<R>();
  // TMA coordinates of the window (0-based column, row, slab l*K + k): x = -3, y = -2
  const int wx = i0 - 4, wy = j0 - 3, wsl = l * K + k;
  bool ok = true;
  if (tid == 0 && !pre) {  // rhog and the first two batches' rhogq stream in during the set-up below
    mbar_expect_tx(&s.mbar[0], QBYTES + RBYTES);
    tma_load_3d(&s.rho[0], &T->rho, wx, wy, wsl, &s.mbar[0]);
    tma_load_4d(&s.stage[0][0][0], &T->q, wx, wy, wsl, 0, &s.mbar[0]);
    if (nbat > 1) {
      mbar_expect_tx(&s.mbar[1], QBYTES);
      tma_load_4d(&s.stage[1][0][0], &T->q, wx, wy, wsl, TB, &s.mbar[1]);
    }
  }

  // this thread's ring cell, at ring position rp (row-major over the ring).  For 16 x 12 tiles the
  // tile cells fill warps 0-5 and the ring border warps 6 (bottom row, left column) and 7 (top row,
  // right column), so a border warp whose cells all lie downstream of the tile (no outflow face
  // into it) skips phase B and leaves its issue slots to the rest (pair 27.7 -> 26.8 ms at gl8 with
  // 4 tracers per batch).  Used by the per-level kernel (BWO) for batches of 16 bytes a cell: with
  // 8 FP32 tracers a batch it measured slower (27.6 against 27.4 ms), and in the persistent kernel
  // the extra registers spill.
  constexpr bool kBorderWarps = BWO && TX == 16 && TY == 12 && TB * sizeof(R) == 16;
  int rp = tid;  // without the border-warp order: thread t takes ring position t (t < NR)
  if (kBorderWarps) {
    if (tid < TX * TY) {
      rp = (tid / TX + 1) * RW + (tid % TX + 1);
    } else {
      const int u = tid - TX * TY, v = u & 31;  // u < 30: warp 6, 32 <= u < 62: warp 7
      if (v >= RW + TY) rp = -1;  // the last two lanes of each border warp
      else if (u < 32) rp = (v < RW) ? v : (v - RW + 1) * RW;                        // y = -1, x = -1
      else rp = (v < RW) ? (TY + 1) * RW + v : (v - RW + 1) * RW + (TX + 1);         // y = TY, x = TX
    }
  }
  const bool ring = kBorderWarps ? rp >= 0 : tid < NR;
  const int x = ring ? rp % RW - 1 : TX + 8, y = ring ? rp / RW - 1 : TY + 8;
  const int ci = i0 + x, cj = j0 + y;
  const int ew = ring ? (y + 2) * WW + (x + 3) : 0;  // window slot of the cell
  const bool in_arr = EDGE ? ring && ci >= 1 && ci <= G && cj >= 1 && cj <= G : ring;
  auto interior = [&](int i, int j) {
    return !EDGE || (i >= I.gmin && i <= I.gmax && j >= I.gmin && j <= I.gmax);
  };
  auto in_tile = [&](int a, int b) { return a >= 0 && a < TX && b >= 0 && b < TY; };
  const bool c_int = in_arr && interior(ci, cj);
  const int bs = (EDGE && in_arr) ? I.bsrc[(size_t)l * I.gall + (cj - 1) * G + (ci - 1)] : -3;
  // Gradient and Qout are formed in the tile for every interior cell, region-boundary cells
  // included: their halo neighbours are in the window, and the fluxes and masks of their seam
  // faces come from k_fast_faces.  The one exception is the corner (gmin, gmin) of a region with
  // the singular point, whose face-5 bounds take the shifted stencil of the singular point; it
  // reads its FP64 values from k_fast_boundary.  (Reading every region-boundary cell's values
  // from that DRAM-resident buffer stalled the edge tiles at every batch barrier.)
  const bool tile_cell = c_int && !(EDGE && sgp && ci == I.gmin && cj == I.gmin);
  const bool active = c_int && in_tile(x, y);  // updated by this thread
  const size_t ccell = in_arr ? (size_t)(cj - 1) * G + (ci - 1) : 0;
  const size_t oc = base + ccell;

  // ---- set-up, tracer-independent: every global load first (one round trip together)
  double Fo[3] = {0.0, 0.0, 0.0}, Fn[3] = {0.0, 0.0, 0.0};  // flux of faces 1-3 (own), 4-6 (owners')
  V4 d4[3];
  R cmn[3] = {R(0.0), R(0.0), R(0.0)};  // owner-side masks of faces 4-6
  const V4 *dupc = (const V4 *)(sizeof(R) == 8 ? (const void *)I.dupc64 : (const void *)I.dupc);
#pragma unroll
  for (int a = 0; a < 3; ++a) d4[a] = V4{R(0.0), R(0.0), R(0.0), R(0.0)};
  double rho_c = 1.0, ra64 = 1.0, wk = 0.0, wk1 = 0.0;
  if (in_arr) {
#pragma unroll
    for (int a = 0; a < 3; ++a) Fo[a] = I.Fg[(size_t)a * n3 + oc], d4[a] = dupc[(size_t)a * n3 + oc];
  }
  if (c_int) {  // owners of faces 4, 5, 6: (i-1, j) face AI, (i-1, j-1) face AIJ, (i, j-1) face AJ
    Fn[0] = I.Fg[oc - 1], cmn[0] = dupc[oc - 1].w;
    Fn[1] = I.Fg[n3 + oc - G - 1], cmn[1] = dupc[n3 + oc - G - 1].w;
    Fn[2] = I.Fg[2 * n3 + oc - G], cmn[2] = dupc[2 * n3 + oc - G].w;
    rho_c = I.rho_in[oc], ra64 = rarea(I, l, ci, cj);
  }
  if (active) wk = fld(I, 3, oc), wk1 = fld(I, 3, oc + slab);
  if (load_cg) {  // level-invariant: loaded once per CTA (horiz_levels)
#pragma unroll
    for (int n = 0; n < 21; ++n)
      cgr[n] = tile_cell ? (sizeof(R) == 8 ? (R)I.cg[((size_t)l * 21 + n) * I.gall + ccell]
                                           : (R)I.cg32[((size_t)l * 21 + n) * I.gall + ccell])
                         : R(0);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (!kBorderWarps || ring) s.dup[a][rp] = d4[a];
  // Courant numbers, upwind sides and the Thuburn outflow sums of the cell
  const R ra32 = (R)ra64;
  R chm[7], omc = R(0.0), rden = R(0.0), zsw = R(1.0);
  unsigned upm = 0;  // bit m: this cell is the upwind cell of its face m (its outflow faces)
#pragma unroll
  for (int m = 0; m < 7; ++m) chm[m] = R(0.0);
  if (c_int) {
    const R rcinv = (R)(1.0 / rho_c);  // by the reciprocal of rho (one division per cell)
    R ch[7];
#pragma unroll
    for (int m = 1; m <= 6; ++m) {
      const R Fm = (R)(m <= 3 ? Fo[m - 1] : Fn[m - 4]);
      ch[m] = ((m <= 3 ? Fm : -Fm) * ra32 * dtf) * rcinv;
      chm[m] = A::mn(ch[m], R(0.0));
      // the owner's mask decides the side: owner upwind where it is 0 (faces 1-3 are this
      // cell's own), the neighbour where it is 1 (faces 4-6, whose owner is the neighbour)
      const bool up = (m <= 3) ? (d4[m - 1].w == R(0.0)) : (cmn[m - 4] != R(0.0));
      upm |= up ? (1u << m) : 0u;
    }
    const R Cin = chm[1] + chm[2] + chm[3] + chm[4] + chm[5] + chm[6];
    const R Cout =
        ch[1] - chm[1] + ch[2] - chm[2] + ch[3] - chm[3] + ch[4] - chm[4] + ch[5] - chm[5] + ch[6] - chm[6];
    zsw = R(0.5) - A::sgn(R(0.5), fabs(Cout) - EPSf);
    omc = R(1.0) - Cin - Cout;
    rden = (R(1.0) - zsw) / (Cout + zsw);
  }
  // the faces this thread fills in qa: its outflow faces between two interior cells (seam faces
  // come from k_fast_seam) that touch a cell of the tile; as owner, its faces 1-3 that touch a
  // tile cell and are seam faces (the seam value) or absent (zero)
  constexpr int DX[7] = {0, 1, 1, 0, -1, -1, 0}, DY[7] = {0, 0, 1, 1, 0, -1, -1};
  unsigned dom = 0, seam_own = 0, zero_own = 0;
  if (c_int) {
#pragma unroll
    for (int m = 1; m <= 6; ++m) {
      const bool need = in_tile(x, y) || in_tile(x + DX[m], y + DY[m]);
      if (need && interior(ci + DX[m], cj + DY[m]) && ((upm >> m) & 1u)) dom |= 1u << m;
    }
  }
  if (EDGE && in_arr && x < TX && y < TY) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int nx = x + DX[a + 1], ny = y + DY[a + 1];
      const bool need = (active) || (in_tile(nx, ny) && interior(ci + DX[a + 1], cj + DY[a + 1]));
      if (!need) continue;
      if (!face_exists(I, ci, cj, a + 1)) zero_own |= 1u << a;
      else if (!c_int || !interior(ci + DX[a + 1], cj + DY[a + 1])) seam_own |= 1u << a;
    }
  }
  // flx_h of the tile cells (FP64), rhog after the horizontal sub-step and the
  // tracer-independent inputs of the vertical sub-step
  if (active) {
    double sum = 0.0;
#pragma unroll
    for (int m = 1; m <= 6; ++m) {
      const double f = cell_flx(I, l, ci, cj, m, sgp, m <= 3 ? Fo[m - 1] : Fn[m - 4], ra64);
      s.flx[m - 1][rp] = f;
      sum = (m == 1) ? f : sum + f;
    }
    const double rho_h = rho_c - sum;
    I.rho_out[oc] = rho_h;
    const double rhinv = 1.0 / rho_h;
    if (sizeof(R) == 8)
      I.vco64[oc] = make_double4(-wk * dt * I.rdgz[k] * rhinv, wk1 * dt * I.rdgz[k] * rhinv, rhinv, wk);
    else
      I.vco[oc] = make_float4((float)(-wk * dt * I.rdgz[k] * rhinv), (float)(wk1 * dt * I.rdgz[k] * rhinv),
                              (float)rhinv, (float)wk);
  }

  // q of the batch in stage[buf] (window slots of this thread), by tracer pairs
  auto load_q = [&](int buf) {
#pragma unroll
    for (int r = 0; r < NSLOT; ++r) {
      const int e = tid + r * NT;
      if (e < NW) {
        const double ri = s.rinv[e];
#pragma unroll
        for (int pp = 0; pp < TP; ++pp)
          s.q2[pp][e] = A::v2((R)(s.stage[buf][2 * pp][e] * ri), (R)(s.stage[buf][2 * pp + 1][e] * ri));
      }
    }
  };
  // ---- 1/rho of the window, then q of the first batch (rho and batch 0 share barrier 0)
  ok = mbar_wait(&s.mbar[0], phase & 1u) && ok;
  phase ^= 1u;
#pragma unroll
  for (int r = 0; r < NSLOT; ++r) {
    const int e = tid + r * NT;
    if (e < NW) {
      const int i = wx + 1 + e % WW, j = wy + 1 + e / WW;  // 1-based cell of the slot
      s.rinv[e] = (i >= 1 && i <= G && j >= 1 && j <= G) ? 1.0 / s.rho[e] : 0.0;
    }
  }
  load_q(0);
  __syncthreads();

  const int st7[7] = {ew, ew + 1, ew + WW + 1, ew + WW, ew - 1, ew - WW - 1, ew - WW};
  const int fslot[7] = {0, rp, rp, rp, rp - 1, rp - RW - 1, rp - RW};  // ring position of face m's owner
  auto cx = [](const V2 &v, int h) { return h ? v.y : v.x; };
  // the FP64 boundary values a singular corner reads (5 per tracer) come from DRAM (bbuf is
  // larger than L2), so the next batch's are prefetched into L1 one batch ahead
  auto prefetch_batch = [&](int tb) {
    const int nt = min(TB, ntr - tb);
    if (EDGE && c_int && !tile_cell) {
#pragma unroll
      for (int tt = 0; tt < TB; ++tt)
        if (tt < nt) {
          const double *bv = bval(I, tb + tt, k, bs);
          asm volatile("prefetch.global.L1 [%0];\n" ::"l"(bv));
          asm volatile("prefetch.global.L1 [%0];\n" ::"l"(bv + 4));
        }
    }
  };
  prefetch_batch(0);
  const R *svals = (const R *)(sizeof(R) == 8 ? (const void *)I.sval64 : (const void *)I.sval);
  for (int t0 = 0, b = 0; t0 < ntr; t0 += TB, ++b) {
    const int ntg = min(TB, ntr - t0);
    if (t0 + TB < ntr) prefetch_batch(t0 + TB);
    // seam faces: their values (k_fast_seam) are copied straight into the owner's qa slots,
    // asynchronously, while phase B runs (no register holds them, and the DRAM latency no
    // longer sits between phase B and its barrier).  Phase B writes no seam slot; the copies
    // are waited for before that barrier.
    if (EDGE && seam_own) {
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if ((seam_own >> a) & 1u) {
          const int sid = I.seam_id[((size_t)l * I.gall + ccell) * 3 + a];
          const R *src = svals + ((size_t)t0 * K + k) * I.ns + sid;
          const size_t tstep = (size_t)K * I.ns;  // next tracer
#pragma unroll
          for (int pp = 0; pp < TP; ++pp) {
            if (2 * pp < ntg) cp_async_elem(&s.qa[pp][a][rp].x, src + (size_t)(2 * pp) * tstep);
            if (2 * pp + 1 < ntg) cp_async_elem(&s.qa[pp][a][rp].y, src + (size_t)(2 * pp + 1) * tstep);
          }
        }
    }
    // ---- (B) per interior ring cell and tracer: gradient and Qout (formed here, or the FP64
    // boundary values at a singular corner), the 4-point bounds of its 6 faces, and the
    // limited value of each of its outflow faces; owners fill their seam and absent faces.  In the
    // border-warp order only cells with an outflow face that touches the tile (dom) take part.
    if (kBorderWarps ? dom != 0u : c_int) {
#pragma unroll
      for (int pp = 0; pp < TP; ++pp) {
        V2 q7[7];
#pragma unroll
        for (int n = 0; n < 7; ++n) q7[n] = s.q2[pp][st7[n]];
        R g[2][3], qmn_c[2], qmx_c[2], lo[2][7], hi[2][7], q0[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          R qs[7];
#pragma unroll
          for (int n = 0; n < 7; ++n) qs[n] = cx(q7[n], h);
          q0[h] = qs[0];
          // bounds of face m: the cell and its neighbours m-1, m, m+1 (cyclic, n0 = n6),
          // mod_src_tracer.f90:152-214
          const R c0 = qs[0], n1 = qs[1], n2 = qs[2], n3 = qs[3], n4 = qs[4], n5 = qs[5], n6 = qs[6];
          const R l12 = A::mn(n1, n2), l34 = A::mn(n3, n4), l56 = A::mn(n5, n6);
          const R h12 = A::mx(n1, n2), h34 = A::mx(n3, n4), h56 = A::mx(n5, n6);
          lo[h][1] = A::mn(c0, A::mn(n6, l12)), hi[h][1] = A::mx(c0, A::mx(n6, h12));
          lo[h][2] = A::mn(c0, A::mn(l12, n3)), hi[h][2] = A::mx(c0, A::mx(h12, n3));
          lo[h][3] = A::mn(c0, A::mn(n2, l34)), hi[h][3] = A::mx(c0, A::mx(n2, h34));
          lo[h][4] = A::mn(c0, A::mn(l34, n5)), hi[h][4] = A::mx(c0, A::mx(h34, n5));
          lo[h][5] = A::mn(c0, A::mn(n4, l56)), hi[h][5] = A::mx(c0, A::mx(n4, h56));
          lo[h][6] = A::mn(c0, A::mn(l56, n1)), hi[h][6] = A::mx(c0, A::mx(h56, n1));
          if (tile_cell) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              R gg = cgr[c * 7] * qs[0];
#pragma unroll
              for (int n = 1; n < 7; ++n) gg = gg + cgr[c * 7 + n] * qs[n];
              g[h][c] = gg;
            }
            // Thuburn outflow bounds (mod_src_tracer.f90:219-282, d = 0): the inflow faces are
            // this cell's faces that are not outflow faces
            R qnmin = c0, qnmax = c0, CQmin = R(0.0), CQmax = R(0.0);
#pragma unroll
            for (int m = 1; m <= 6; ++m) {
              const bool in = !((upm >> m) & 1u);
              const R qmn = in ? lo[h][m] : BIGf, qmx = in ? hi[h][m] : -BIGf;
              qnmin = A::mn(qnmin, qmn);
              qnmax = A::mx(qnmax, qmx);
              CQmin = (m == 1) ? chm[1] * qmn : CQmin + chm[m] * qmn;
              CQmax = (m == 1) ? chm[1] * qmx : CQmax + chm[m] * qmx;
            }
            qmn_c[h] = (c0 - CQmax - qnmax * omc) * rden + c0 * zsw;
            qmx_c[h] = (c0 - CQmin - qnmin * omc) * rden + c0 * zsw;
          } else if (EDGE) {  // singular corner: the FP64 boundary values (k_fast_boundary)
            const bool okt = 2 * pp + h < ntg;
            const double *bv = bval(I, okt ? t0 + 2 * pp + h : t0, k, bs);
            g[h][0] = okt ? (R)bv[0] : R(0.0);
            g[h][1] = okt ? (R)bv[1] : R(0.0);
            g[h][2] = okt ? (R)bv[2] : R(0.0);
            qmn_c[h] = okt ? (R)bv[3] : R(0.0);
            qmx_c[h] = okt ? (R)bv[4] : R(0.0);
          }
        }
        // limited values of the outflow faces (remap with the upwind gradient, clipped to the
        // face's 4-point bounds, then to the upwind cell's Qout; :378-410)
#pragma unroll
        for (int m = 1; m <= 6; ++m) {
          if (!((dom >> m) & 1u)) continue;
          const int a = (m - 1) % 3;
          const V4 dv = s.dup[a][fslot[m]];
          R v[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            R w = q0[h];
            w = w + g[h][0] * dv.x;
            w = w + g[h][1] * dv.y;
            w = w + g[h][2] * dv.z;
            w = A::mn(A::mx(w, lo[h][m]), hi[h][m]);
            v[h] = A::mx(A::mn(w, qmx_c[h]), qmn_c[h]);
          }
          s.qa[pp][a][fslot[m]] = A::v2(v[0], v[1]);
        }
      }
    }
    if (EDGE && zero_own) {
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if ((zero_own >> a) & 1u) {
#pragma unroll
          for (int pp = 0; pp < TP; ++pp) s.qa[pp][a][rp] = A::v2(R(0.0), R(0.0));
        }
    }
    cp_async_wait_all();  // this thread's seam copies
    __syncthreads();
    // ---- (D) horizontal update of the tile cells (FP64): rhogq after the horizontal sub-step.
    // For tile rows of 16 or 32 cells, compact: thread t updates tile cell t (every operand is in
    // shared memory, found by the cell's ring position), so the update runs on TX*TY/32 warps with
    // whole rows per warp instead of on all of the ring's warps with their ring lanes idle (27.7
    // against 28.4 ms at gl8 for 16 x 12).  Other widths keep the ring thread (with 14-cell rows a
    // compact warp's stores straddle three rows: 29.0 against 27.9 ms).
    constexpr bool kCompactD = (TX == 16 || TX == 32);
    if (kCompactD ? tid < TX * TY : active) {
      const int dx = kCompactD ? tid % TX : x, dy = kCompactD ? tid / TX : y;
      const int di = i0 + dx, dj = j0 + dy;
      const bool dact = !kCompactD || !EDGE || (di <= I.gmax && dj <= I.gmax);  // a tile cell is >= gmin
      const int dp = kCompactD ? (dy + 1) * RW + (dx + 1) : rp;  // ring position
      const int dew = kCompactD ? (dy + 2) * WW + (dx + 3) : ew;  // window slot
      const size_t doc = kCompactD ? base + (size_t)(dj - 1) * G + (di - 1) : oc;
      double fx[7];
#pragma unroll
      for (int m = 1; m <= 6; ++m) fx[m] = dact ? s.flx[m - 1][dp] : 0.0;
#pragma unroll
      for (int pp = 0; pp < TP; ++pp) {
        if (!dact) break;
        const V2 f1 = s.qa[pp][0][dp], f2 = s.qa[pp][1][dp], f3 = s.qa[pp][2][dp];
        const V2 f4 = s.qa[pp][0][dp - 1], f5 = s.qa[pp][1][dp - RW - 1], f6 = s.qa[pp][2][dp - RW];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int tt = 2 * pp + h;
          if (tt >= ntg) break;
          const size_t o = (size_t)(t0 + tt) * n3 + doc;
          const double Qin = s.stage[b & 1][tt][dew];
          const R qa[7] = {R(0.0), cx(f1, h), cx(f2, h), cx(f3, h), cx(f4, h), cx(f5, h), cx(f6, h)};
          double sum = fx[1] * (double)qa[1];
#pragma unroll
          for (int m = 2; m <= 6; ++m) sum = sum + fx[m] * (double)qa[m];
          I.Q_out[o] = Qin - sum;
        }
      }
    }
    // ---- (A) q of the next batch, whose copy streamed in during (B)
    if (b + 1 < nbat) {
      const int nb1 = (b + 1) & 1;
      ok = mbar_wait(&s.mbar[nb1], (phase >> nb1) & 1u) && ok;
      phase ^= 1u << nb1;
      load_q(nb1);
    }
    __syncthreads();
    // every read of stage[b & 1] is done: batch b + 2 streams into it, or, for an even count of
    // batches, the next level's batch b + 2 - nbat (with its rhog for the first: the current
    // level's rhog window was last read when 1/rhog was formed in the set-up)
    if (tid == 0 && b + 2 < nbat) {
      mbar_expect_tx(&s.mbar[b & 1], QBYTES);
      tma_load_4d(&s.stage[b & 1][0][0], &T->q, wx, wy, wsl, (b + 2) * TB, &s.mbar[b & 1]);
    } else if (tid == 0 && knext >= 0) {
      const int wsn = l * K + knext;
      if (b + 2 == nbat) {
        mbar_expect_tx(&s.mbar[0], QBYTES + RBYTES);
        tma_load_3d(&s.rho[0], &T->rho, wx, wy, wsn, &s.mbar[0]);
        tma_load_4d(&s.stage[0][0][0], &T->q, wx, wy, wsn, 0, &s.mbar[0]);
      } else {
        mbar_expect_tx(&s.mbar[1], QBYTES);
        tma_load_4d(&s.stage[1][0][0], &T->q, wx, wy, wsn, TB, &s.mbar[1]);
      }
    }
  }
  if (!ok && tid == 0) atomicOr(I.err, 1);
  return ok;
}

// work item (tile, level) in the form its position needs (uniform over the CTA)
template <int TX, int TY, int TB, typename R>
__device__ __forceinline__ bool horiz_tile(const FastInst I, const TileMaps *T, const int tile, const int k,
                                           TileSmem<TX, TY, TB, R> &s, unsigned &phase) {
  R cgr[21];
  const int tr = tile % (I.ntx * I.nty);
  if (edge_tile<TX, TY>(I, I.gmin + (tr % I.ntx) * TX, I.gmin + (tr / I.ntx) * TY))
    return horiz_item<TX, TY, TB, R, true>(I, T, tile, k, s, phase, cgr);
  return horiz_item<TX, TY, TB, R, false>(I, T, tile, k, s, phase, cgr);
}

// levels [k0, k1) of a tile in one CTA: the gradient coefficients stay in registers, and (for an
// even count of tracer batches) each level's first copies are issued as the previous level
// frees the stage buffers
template <int TX, int TY, int TB, typename R, bool EDGE>
__device__ __forceinline__ void horiz_levels(const FastInst &I, const TileMaps *T, const int tile, const int k0,
                                             const int k1, TileSmem<TX, TY, TB, R> &s, unsigned &phase) {
  R cgr[21];
  const int nbat = (I.ntr + TB - 1) / TB;
  const bool chain = nbat >= 2 && (nbat & 1) == 0;
  for (int k = k0; k < k1; ++k) {
    const bool ok = horiz_item<TX, TY, TB, R, EDGE, true>(I, T, tile, k, s, phase, cgr, k == k0,
                                                          chain && k > k0, chain && k + 1 < k1 ? k + 1 : -1);
    if (__syncthreads_or(!ok)) break;  // also: this level's shared data is read before the next set-up
  }
}

template <int TX, int TY, int TB, typename R>
__device__ __forceinline__ TileSmem<TX, TY, TB, R> &tile_smem(unsigned char *raw) {
  // The dynamic allocation carries 128 bytes of slack for this alignment (TMA destinations).
  // The offset is applied to the shared array itself, not through an integer round trip, so
  // the compiler keeps the shared address space: every access of the tile is an LDS/STS with a
  // 32-bit address instead of a generic load with a 64-bit one (5% of the kernel's time).
  unsigned char *a = raw + ((128u - (smem_u32(raw) & 127u)) & 127u);
  return *reinterpret_cast<TileSmem<TX, TY, TB, R> *>(a);
}

// Batches of instances: persistent, one wave of CTAs; each takes the next work item
// (instance, level, tile; tiles fastest) from a counter that starts at zero, so CTAs that
// drew cheap items take more (as fast as one CTA per item; a static stride was 9% slower).
template <int TX, int TY, int TB, typename R>
__global__ void __launch_bounds__(TileGeo<TX, TY>::NT, (sizeof(R) == 8 ? 1 : 2))
    k_fast_horiz(const __grid_constant__ MultiInst M, const __grid_constant__ MultiMaps T, long long nwork) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto &s = tile_smem<TX, TY, TB, R>(smem_raw);
  __shared__ long long s_item;
  tile_smem_init(s);
  unsigned phase = 0;
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(M.inst[0].work_next, 1ULL);
    __syncthreads();
    long long wi = s_item;
    if (wi >= nwork) break;
    const int ii =
        find_inst(M, wi, [](const FastInst &J) { return (long long)(J.l1 - J.l0) * J.ntx * J.nty * (J.K - 2); });
    const int tpr = M.inst[ii].ntx * M.inst[ii].nty, ntl = (M.inst[ii].l1 - M.inst[ii].l0) * tpr;
    const int tile = M.inst[ii].l0 * tpr + (int)(wi % ntl), k = 1 + (int)(wi / ntl);
    bool ok;
    switch (ii) {
      case 0: ok = horiz_tile<TX, TY, TB, R>(M.inst[0], &T.m[0], tile, k, s, phase); break;
      case 1: ok = horiz_tile<TX, TY, TB, R>(M.inst[1], &T.m[1], tile, k, s, phase); break;
      case 2: ok = horiz_tile<TX, TY, TB, R>(M.inst[2], &T.m[2], tile, k, s, phase); break;
      default: ok = horiz_tile<TX, TY, TB, R>(M.inst[3], &T.m[3], tile, k, s, phase); break;
    }
    // the next item's data overwrite this item's shared data; s_item is reread
    if (__syncthreads_or(!ok)) break;
  }
}

// one grid: one CTA per (tile, kLevelsPerCta consecutive levels) (grid x = level block, y = tile:
// a tile's level blocks run side by side, so its level-invariant coefficients are read from L2
// by all but the first, and a CTA keeps them in registers over its levels)
constexpr int kLevelsPerCta = 8;
template <int TX, int TY, int TB, typename R>
__global__ void __launch_bounds__(TileGeo<TX, TY>::NT, (sizeof(R) == 8 ? 1 : 2))
    k_fast_horiz1(const __grid_constant__ FastInst I, const __grid_constant__ TileMaps T) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto &s = tile_smem<TX, TY, TB, R>(smem_raw);
  tile_smem_init(s);
  unsigned phase = 0;
  const int tile = I.l0 * I.ntx * I.nty + (int)blockIdx.y, tr = (int)blockIdx.y % (I.ntx * I.nty);
  const int k0 = 1 + (int)blockIdx.x * kLevelsPerCta, k1 = min(k0 + kLevelsPerCta, I.K - 1);
  if (edge_tile<TX, TY>(I, I.gmin + (tr % I.ntx) * TX, I.gmin + (tr / I.ntx) * TY))
    horiz_levels<TX, TY, TB, R, true>(I, &T, tile, k0, k1, s, phase);
  else
    horiz_levels<TX, TY, TB, R, false>(I, &T, tile, k0, k1, s, phase);
}

// ---- vertical sub-step: one thread per (interior column, TV tracers), streaming the
// levels with the limiter two levels behind and the next two levels' inputs in flight; FP32
// limiter, FP64 update.  rhogq after the horizontal sub-step is read from (and the result
// written to) Q_out; the threads of the first tracer group also finish rhog.
// The tracer groups of a column block are consecutive blocks, so they run together and
// share the per-level inputs (vco) in L2.
// The column kernel's inputs stream through a shared-memory ring of kVertStages levels, filled
// by each thread's own cp.async copies (no barrier: a thread reads only what it copied), so
// kVertStages - 1 levels of every column are in flight without holding registers.  With the
// level loop below (peeled first levels, fixed window slots, 32-bit offsets, no per-tracer
// branches) the kernel runs without spills: 8.6 -> 6.7 ms per gl8 step, the same results.
constexpr int kVertStages = 3;
template <int TV, typename R>
struct VertRing {
  using V4 = typename std::conditional<sizeof(R) == 8, double4, float4>::type;
  double q[kVertStages][TV][256];
  V4 v[kVertStages][256];
  double r[kVertStages][256];
};
template <int TV, typename R>
__device__ __forceinline__ void vert_block(const FastInst &I, long long blk) {
  using A = Arith<R>;
  using V4 = typename std::conditional<sizeof(R) == 8, double4, float4>::type;
  static_assert(kVertStages == 3, "ring slot = level % 3 = register window slot");
  extern __shared__ __align__(16) unsigned char vraw[];
  VertRing<TV, R> &ring = *reinterpret_cast<VertRing<TV, R> *>(vraw);
  const int th = threadIdx.x;
  const int ngr = (I.ntr + TV - 1) / TV;
  const int t0 = (int)(blk % ngr) * TV;
  const int n = I.gmax - I.gmin + 1;
  const long long col = (blk / ngr) * blockDim.x + th;
  if (col >= (long long)(I.l1 - I.l0) * n * n) return;
  const int l = I.l0 + (int)(col / ((long long)n * n)), r = (int)(col % ((long long)n * n));
  const int i = I.gmin + r % n, j = I.gmin + r / n;
  const int K = I.K;
  const unsigned slab = (unsigned)I.gall;
  const size_t tstride = (size_t)I.lall * K * slab;
  const size_t cbase = (size_t)l * K * slab + (size_t)(j - 1) * I.G + (i - 1);
  double *Q = I.Q_out + (size_t)t0 * tstride + cbase;
  // 32-bit offsets from Q: tracer tt of the group (a partial last group repeats its first
  // tracer: the same values computed and stored twice by this thread) plus the level's
  unsigned tof[TV];
#pragma unroll
  for (int tt = 0; tt < TV; ++tt) tof[tt] = (t0 + tt < I.ntr) ? (unsigned)(tt * tstride) : 0u;
  double *RH = I.rho_out + cbase;
  const V4 *V = (const V4 *)(sizeof(R) == 8 ? (const void *)I.vco64 : (const void *)I.vco) + cbase;
  const bool dens = t0 == 0;
  const double dt = I.dt;
  // level k's values live in slot k % 3 of each window, in registers and in the ring (the level
  // loop is unrolled three times with the slots fixed per copy: no copies between levels)
  R ck1w[3] = {R(0.0), R(0.0), R(0.0)}, ck2w[3] = {R(0.0), R(0.0), R(0.0)}, wf[3] = {R(0.0), R(0.0), R(0.0)};
  double rh[3] = {0.0, 0.0, 0.0};
  double Qh[TV][3];
  R qv[TV][3], qmn_km1[TV], qmx_km1[TV];
  double fu_last[TV];  // w qh of the face below the level being finished (the flux of the level below)
  auto issue = [&](int kq) {  // level kq's inputs into ring slot kq % 3
    if (kq <= K - 2) {
      const int sl = kq % kVertStages;
      const unsigned o = (unsigned)kq * slab;
#pragma unroll
      for (int tt = 0; tt < TV; ++tt) cp_async_elem(&ring.q[sl][tt][th], Q + (tof[tt] + o));
#pragma unroll
      for (int h = 0; h < (int)(sizeof(V4) / 16); ++h)
        cp_async_16((unsigned char *)&ring.v[sl][th] + 16 * h, (const unsigned char *)(V + o) + 16 * h);
      if (dens) cp_async_elem(&ring.r[sl][th], RH + o);
    }
    cp_async_commit();
  };
  issue(1);
  issue(2);
  // level k in slot S0 = k % 3 (S1, S2: levels k-1, k-2).  KIND 1: the first level (and the ghost
  // level below it, q(kmin-1) = q(kmin)); 2: the second (Qout of level 1, face 1 unlimited by
  // the level below); 3: the third (level 1 final, also into the ghost level); 4: the rest.
  auto level = [&](const int k, auto s0, auto kind) {
    constexpr int S0 = decltype(s0)::value, S1 = (S0 + 2) % 3, S2 = (S0 + 1) % 3;
    constexpr int KIND = decltype(kind)::value;
    cp_async_wait<kVertStages - 2>();  // level k's group is complete
    const V4 c = ring.v[S0][th];
    double Qk[TV];
#pragma unroll
    for (int tt = 0; tt < TV; ++tt) Qk[tt] = ring.q[S0][tt][th];
    const double rk = dens ? ring.r[S0][th] : 0.0;
    issue(k + 2);  // into the ring slot of level k - 1, read in the previous level
    ck1w[S0] = c.x, ck2w[S0] = c.y, wf[S0] = c.w, rh[S0] = rk;
    if (KIND == 1) {
#pragma unroll
      for (int tt = 0; tt < TV; ++tt) {
        Qh[tt][S0] = Qk[tt];
        qv[tt][S1] = qv[tt][S0] = (R)(Qk[tt] * (double)c.z);
        fu_last[tt] = 0.0;  // qh(kmin) = 0 at the ground face
      }
      return;
    }
    // Qout of level k-1 from q at k-2, k-1, k; the face k-1 between levels k-2 and k-1
    const VLim<R> vp = vlim_params<R>(ck1w[S1], ck2w[S1], ck1w[S0]);
    const int f = k - 1;
    const R af = (R)I.afact[f], bf = (R)I.bfact[f];
    const double dtrdz = dt * I.rdgz[k - 2];
    const unsigned os = (unsigned)(k - 2) * slab;
#pragma unroll
    for (int tt = 0; tt < TV; ++tt) {
      Qh[tt][S0] = Qk[tt];
      qv[tt][S0] = (R)(Qk[tt] * (double)c.z);
      R Qmin, Qmax;
      vlim_qout(vp, qv[tt][S2], qv[tt][S1], qv[tt][S0], Qmin, Qmax);
      R qh = af * qv[tt][S1] + bf * qv[tt][S2];
      if (KIND >= 3)
        qh = vp.infl * A::mx(A::mn(qh, qmx_km1[tt]), qmn_km1[tt]) + (R(1.0) - vp.infl) * A::mx(A::mn(qh, Qmax), Qmin);
      const double fu = (double)wf[S1] * (double)qh;
      if (KIND >= 3) {  // level k-2 is final once faces k-2 and k-1 are
        const double Qn = Qh[tt][S2] - (fu - fu_last[tt]) * dtrdz;
        Q[tof[tt] + os] = Qn;
        if (KIND == 3) Q[tof[tt]] = Qn;
      }
      fu_last[tt] = fu;
      qmn_km1[tt] = Qmin;
      qmx_km1[tt] = Qmax;
    }
    if (KIND >= 3 && dens) {
      const double rn = rh[S2] - ((double)wf[S1] - (double)wf[S2]) * dtrdz;
      RH[os] = rn;
      if (KIND == 3) RH[0] = rn;
    }
  };
  using C0 = std::integral_constant<int, 0>;
  using C1 = std::integral_constant<int, 1>;
  using C2 = std::integral_constant<int, 2>;
  using K1 = std::integral_constant<int, 1>;
  using K2 = std::integral_constant<int, 2>;
  using K3 = std::integral_constant<int, 3>;
  using K4 = std::integral_constant<int, 4>;
  level(1, C1{}, K1{});
  if (K - 2 >= 2) level(2, C2{}, K2{});
  if (K - 2 >= 3) level(3, C0{}, K3{});
  int k = 4;
#pragma unroll 1
  for (; k + 2 <= K - 2; k += 3) {
    level(k, C1{}, K4{});
    level(k + 1, C2{}, K4{});
    level(k + 2, C0{}, K4{});
  }
  if (k <= K - 2) level(k++, C1{}, K4{});
  if (k <= K - 2) level(k++, C2{}, K4{});
  // ---- drain: levels K-3 and K-2 (faces K-2 and K-1); ghost level above: q(kmax+1) = q(kmax)
  auto drain = [&](auto sl) {
    constexpr int SL = decltype(sl)::value, SP = (SL + 2) % 3;  // slots of levels K-2, K-3
    const int kk = K - 1;
    const R wk1 = (R)fld(I, 3, cbase + (size_t)kk * slab);
    const R c1top = (R)(-(double)wk1 * dt * I.rdgz[kk] / I.rho_in[cbase + (size_t)kk * slab]);
    const VLim<R> vd = vlim_params<R>(ck1w[SL], ck2w[SL], c1top);  // level K-2 with q(K-1) := q(K-2)
    const int f = K - 2;
    const R af = (R)I.afact[f], bf = (R)I.bfact[f];
    const R ak = (R)I.afact[kk], bk = (R)I.bfact[kk];
#pragma unroll
    for (int tt = 0; tt < TV; ++tt) {
      R Qmin, Qmax;
      vlim_qout(vd, qv[tt][SP], qv[tt][SL], qv[tt][SL], Qmin, Qmax);
      R qh = af * qv[tt][SL] + bf * qv[tt][SP];
      if (f >= 2)
        qh = vd.infl * A::mx(A::mn(qh, qmx_km1[tt]), qmn_km1[tt]) + (R(1.0) - vd.infl) * A::mx(A::mn(qh, Qmax), Qmin);
      double *Qt = Q + tof[tt];
      const double fm = (double)wf[SL] * (double)qh;  // face K-2
      if (K - 3 >= 1) {
        const int L = K - 3;
        const double Qn = Qh[tt][SP] - (fm - fu_last[tt]) * (dt * I.rdgz[L]);
        Qt[(size_t)L * slab] = Qn;
        if (L == 1) Qt[0] = Qn;
      }
      // top face K-1: unlimited
      const R qtop = ak * qv[tt][SL] + bk * qv[tt][SL];
      const double fu = (double)wk1 * (double)qtop;
      const double Qn = Qh[tt][SL] - (fu - fm) * (dt * I.rdgz[K - 2]);
      Qt[(size_t)(K - 2) * slab] = Qn;
      Qt[(size_t)(K - 1) * slab] = Qn;
      if (K - 2 == 1) Qt[0] = Qn;
    }
    if (dens) {
      if (K - 3 >= 1) {
        const int L = K - 3;
        const double rn = rh[SP] - ((double)wf[SL] - (double)wf[SP]) * (dt * I.rdgz[L]);
        RH[(size_t)L * slab] = rn;
        if (L == 1) RH[0] = rn;
      }
      const double rn = rh[SL] - ((double)wk1 - (double)wf[SL]) * (dt * I.rdgz[K - 2]);
      RH[(size_t)(K - 2) * slab] = rn;
      RH[(size_t)(K - 1) * slab] = rn;
      if (K - 2 == 1) RH[0] = rn;
    }
  };
  switch ((K - 2) % 3) {
    case 0: drain(C0{}); break;
    case 1: drain(C1{}); break;
    default: drain(C2{}); break;
  }
  cp_async_wait_all();  // the trailing groups are empty; nothing is left in flight at exit
}
template <int TV, typename R>
__global__ void __launch_bounds__(256, 2) k_fast_vert1(FastInst I) {
  vert_block<TV, R>(I, blockIdx.x);
}

template <int TV, typename R>
__global__ void __launch_bounds__(256, 2) k_fast_vert(const __grid_constant__ MultiInst M) {
  // blocks of an instance: (tracer group fastest, column block)
  long long blk = blockIdx.x;
  const int ii = find_inst(M, blk, [](const FastInst &J) {
    const long long nc = (long long)(J.l1 - J.l0) * (J.gmax - J.gmin + 1) * (J.gmax - J.gmin + 1);
    return (long long)((J.ntr + TV - 1) / TV) * ((nc + 255) / 256);
  });
  switch (ii) {
    case 0: vert_block<TV, R>(M.inst[0], blk); break;
    case 1: vert_block<TV, R>(M.inst[1], blk); break;
    case 2: vert_block<TV, R>(M.inst[2], blk); break;
    case 3: vert_block<TV, R>(M.inst[3], blk); break;
    default: break;
  }
}

// ---- the two pole centres, FP64: one CTA per (pole, tracer), one thread per level ----------
// The horizontal sub-step of every level, then the vertical one of the column: its Qout of a
// level needs only q and the Courant numbers, so every stage is level-parallel.  Each value
// takes the operations of the column form; this file allows FMA contraction, so results
// can differ from that form at FP64 rounding.
template <int KMAX>
__global__ void __launch_bounds__(KMAX) k_fast_pole(const __grid_constant__ MultiInst M) {
  long long tl = blockIdx.x;
  const int ii = find_inst(M, tl, [](const FastInst &J) { return J.poles ? (long long)kLallPl * J.ntr : 0LL; });
  if (ii < 0) return;  // whole CTA
  const FastInst &I = M.inst[ii];
  const int t = (int)tl;
  const int p = t % kLallPl, tr = t / kLallPl;
  const int K = I.K, k = threadIdx.x;
  const int kmin = 1, kmax = K - 2;
  const size_t toff = (size_t)tr * kLallPl * K * kGallPl;
  const double rarea = I.GMTR_p_pl[((size_t)(P_RAREA - 1) * kLallPl + p) * kGallPl];
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  __shared__ double sQh[KMAX], srh[KMAX], sq[KMAX], sqh[KMAX], sck1[KMAX], sck2[KMAX], sQmn[KMAX], sQmx[KMAX],
      sinfl[KMAX];
  // ---- horizontal sub-step of level k
  if (k >= kmin && k <= kmax) {
    const size_t off = ((size_t)p * K + k) * kGallPl;
    double flux[7], xc[7][3];
    pole_faces(I, p, k, flux, xc);
    double q[7], g[7][3], Qmn[7], Qmx[7];
    for (int v = 1; v <= 6; ++v) q[v] = I.Q_in_pl[toff + off + v - 1] / I.rho_in_pl[off + v - 1];
    const double *bc = bval(I, tr, k, I.nb - 2 + p);
    for (int x = 0; x < 3; ++x) g[1][x] = bc[x];
    Qmn[1] = bc[3], Qmx[1] = bc[4];
    for (int v = 2; v <= 6; ++v) {
      const double *br = bval(I, tr, k, I.pole_ring_b[p * 5 + (v - 2)]);
      for (int x = 0; x < 3; ++x) g[v][x] = br[x];
      Qmn[v] = br[3], Qmx[v] = br[4];
    }
    double sum = 0.0, rsum = 0.0;
    for (int v = 2; v <= 6; ++v) {
      const double flx = flux[v] * rarea * I.dt;
      const double ch = flx / I.rho_in_pl[off];
      const double c = 0.5 - fsg(0.5, ch - EPS);
      double vu = q[v], vs = q[1];
      for (int x = 0; x < 3; ++x) vu = vu + g[v][x] * (xc[v][x] - I.GRD_x_pl[((size_t)x * kLallPl + p) * kGallPl + v - 1]);
      for (int x = 0; x < 3; ++x) vs = vs + g[1][x] * (xc[v][x] - I.GRD_x_pl[((size_t)x * kLallPl + p) * kGallPl]);
      double a = c * vu + (1.0 - c) * vs;
      const int vp = (v == 6) ? 2 : v + 1, vm = (v == 2) ? 6 : v - 1;
      const double lo = mn64(mn64(mn64(q[1], q[v]), q[vm]), q[vp]);
      const double hi = mx64(mx64(mx64(q[1], q[v]), q[vm]), q[vp]);
      const double i1min = c * lo + (1.0 - c) * BIG, i1max = c * hi + (1.0 - c) * (-BIG);
      const double i2min = c * BIG + (1.0 - c) * lo, i2max = c * (-BIG) + (1.0 - c) * hi;
      a = c * mn64(mx64(a, i1min), i1max) + (1.0 - c) * mn64(mx64(a, i2min), i2max);
      a = c * mx64(mn64(a, Qmx[v]), Qmn[v]) + (1.0 - c) * mx64(mn64(a, Qmx[1]), Qmn[1]);
      if (v == 2) sum = flx * a, rsum = flx;
      else sum = sum + flx * a, rsum = rsum + flx;
    }
    sQh[k] = I.Q_in_pl[toff + off] - sum;
    srh[k] = I.rho_in_pl[off] - rsum;
  }
  __syncthreads();
  // ---- vertical sub-step of the pole column (FP64, region form, as the plain path)
  auto W = [&](int kk) { return fld_pl(I, 3, ((size_t)p * K + kk) * kGallPl); };
  if (k < K) {
    double c1 = 0.0, c2 = 0.0;
    if (k >= kmin && k <= kmax) {
      c1 = -W(k) * I.dt * I.rdgz[k] / srh[k];
      c2 = W(k + 1) * I.dt * I.rdgz[k] / srh[k];
      sq[k] = sQh[k] / srh[k];
    }
    if (k == K - 1) c1 = -W(K - 1) * I.dt * I.rdgz[K - 1] / I.rho_in_pl[((size_t)p * K + K - 1) * kGallPl];
    sck1[k] = c1, sck2[k] = c2;
  }
  __syncthreads();
  if (k == 0) sq[0] = sq[kmin];
  if (k == K - 1) sq[K - 1] = sq[kmax];
  __syncthreads();
  if (k >= kmin && k <= kmax + 1 && k < K) sqh[k] = I.afact[k] * sq[k] + I.bfact[k] * sq[k - 1];
  if (k >= kmin && k <= kmax) {  // Qout of level k
    const double infl = 0.5 - fsg(0.5, sck1[k]);
    const double infu = 0.5 + fsg(0.5, sck1[k + 1]);
    const double qk = sq[k], qm = sq[k - 1], qp = sq[k + 1];
    const double minL = mn64(qk, qm) + (1.0 - infl) * BIG, minU = mn64(qk, qp) + (1.0 - infu) * BIG;
    const double maxL = mx64(qk, qm) - (1.0 - infl) * BIG, maxU = mx64(qk, qp) - (1.0 - infu) * BIG;
    const double qnmin = mn64(mn64(minL, minU), qk), qnmax = mx64(mx64(maxL, maxU), qk);
    const double Cin = infl * sck1[k] + infu * sck2[k], Cout = (1.0 - infl) * sck1[k] + (1.0 - infu) * sck2[k];
    const double CQmax = infl * sck1[k] * maxL + infu * sck2[k] * maxU;
    const double CQmin = infl * sck1[k] * minL + infu * sck2[k] * minU;
    const double zerosw = 0.5 - fsg(0.5, fabs(Cout) - EPS);
    sQmn[k] = ((qk - qnmax) + qnmax * (Cin + Cout) - CQmax) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
    sQmx[k] = ((qk - qnmin) + qnmin * (Cin + Cout) - CQmin) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
    sinfl[k] = infl;
  }
  __syncthreads();
  // limited face values of faces kmin+1 .. kmax (bounds of the levels on both sides)
  double hk = 0.0;
  const bool lim = k >= kmin + 1 && k <= kmax;
  if (lim) {
    const double h = sqh[k], infl = sinfl[k];
    hk = infl * mx64(mn64(h, sQmx[k - 1]), sQmn[k - 1]) + (1.0 - infl) * mx64(mn64(h, sQmx[k]), sQmn[k]);
  }
  __syncthreads();
  if (lim) sqh[k] = hk;
  __syncthreads();
  if (k >= kmin && k <= kmax) {
    const double Qn = sQh[k] - (W(k + 1) * sqh[k + 1] - W(k) * sqh[k]) * I.dt * I.rdgz[k];
    double *Qo = I.Q_out_pl + toff + (size_t)p * K * kGallPl;
    Qo[(size_t)k * kGallPl] = Qn;
    if (k == kmin) Qo[0] = Qn;
    if (k == kmax) Qo[(size_t)(K - 1) * kGallPl] = Qn;
    if (tr == 0) {
      const double rn = srh[k] - (W(k + 1) - W(k)) * I.dt * I.rdgz[k];
      double *Ro = I.rho_out_pl + (size_t)p * K * kGallPl;
      Ro[(size_t)k * kGallPl] = rn;
      if (k == kmin) Ro[0] = rn;
      if (k == kmax) Ro[(size_t)(K - 1) * kGallPl] = rn;
    }
  }
}

// ---- halo points no list writes keep their input values (the reference never touches them)
__global__ void k_fast_carry(const __grid_constant__ MultiInst M) {
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = find_inst(M, tid, [](const FastInst &J) { return (long long)J.ncarry * J.K; });
  if (ii < 0) return;
  const FastInst &I = M.inst[ii];
  const int p = I.carry[tid % I.ncarry], k = (int)(tid / I.ncarry);
  if (p < 0 || !owns_point(I, p)) return;
  const int l = p / I.gall, c = p % I.gall;
  const size_t off = ((size_t)l * I.K + k) * I.gall + c, tstride = (size_t)I.lall * I.K * I.gall;
  I.rho_out[off] = I.rho_in[off];
  for (int t = 0; t < I.ntr; ++t) I.Q_out[(size_t)t * tstride + off] = I.Q_in[(size_t)t * tstride + off];
}

// ---------------------------------------------------------------------------------------
// TMA descriptors of the tile windows.  cuTensorMapEncodeTiled is a driver-API function; it is
// reached through the runtime's driver entry point, so the library links only cudart.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
    cudaGetLastError();
  });
  return fn;
}

// rhogq_in as (i, j, l*K + k, tracer) with box (WW, WH, 1, TB) and rhog_in as (i, j, l*K + k)
// with box (WW, WH, 1); out-of-range elements of a box are filled with zeros.
static cudaError_t tile_maps(const FastInst &I, int WW, int WH, int TB, TileMaps &T) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  const cuuint64_t G = (cuuint64_t)I.G, S = (cuuint64_t)I.lall * I.K;
  const cuuint64_t dq[4] = {G, G, S, (cuuint64_t)I.ntr};
  const cuuint64_t sq[3] = {G * 8, G * G * 8, S * G * G * 8};
  const cuuint32_t bq[4] = {(cuuint32_t)WW, (cuuint32_t)WH, 1, (cuuint32_t)TB};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(&T.q, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)I.Q_in, dq, sq, bq, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  r = enc(&T.rho, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)I.rho_in, dq, sq, bq, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  return cudaSuccess;
}

template <int TX, int TY, int TB, bool ONE, typename R>
static cudaError_t launch_tile_n(const MultiInst &M, cudaStream_t st) {
  const int smem = (int)sizeof(TileSmem<TX, TY, TB, R>) + 128;  // + slack for the 128-byte alignment
  constexpr int NT = TileGeo<TX, TY>::NT;
  static int per_sm[64] = {};  // resident CTAs per SM, per device (set up once, outside any capture)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!per_sm[dev]) {
    int occ = 0;
    if (ONE) {
      e = cudaFuncSetAttribute(k_fast_horiz1<TX, TY, TB, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fast_horiz1<TX, TY, TB, R>, NT, smem);
    } else {
      e = cudaFuncSetAttribute(k_fast_horiz<TX, TY, TB, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fast_horiz<TX, TY, TB, R>, NT, smem);
    }
    if (e != cudaSuccess) return e;
    per_sm[dev] = occ > 0 ? occ : 1;
  }
  int nsm = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  MultiMaps T;
  for (int i = 0; i < M.n; ++i) {
    e = tile_maps(M.inst[i], TileGeo<TX, TY>::WW, TileGeo<TX, TY>::WH, TB, T.m[i]);
    if (e != cudaSuccess) return e;
  }
  long long nwork = 0;
  for (int i = 0; i < M.n; ++i)
    nwork += (long long)(M.inst[i].l1 - M.inst[i].l0) * M.inst[i].ntx * M.inst[i].nty * (M.inst[i].K - 2);
  if (ONE) {
    const FastInst &I = M.inst[0];
    if ((long long)(I.l1 - I.l0) * I.ntx * I.nty > 65535) return cudaErrorInvalidConfiguration;  // grid y
    k_fast_horiz1<TX, TY, TB, R>
        <<<dim3((unsigned)((I.K - 2 + kLevelsPerCta - 1) / kLevelsPerCta), (unsigned)((I.l1 - I.l0) * I.ntx * I.nty)),
           NT, smem, st>>>(I, T.m[0]);
  } else {
    const long long grid = nwork < (long long)nsm * per_sm[dev] ? nwork : (long long)nsm * per_sm[dev];
    e = cudaMemsetAsync(M.inst[0].work_next, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_fast_horiz<TX, TY, TB, R><<<(unsigned)grid, NT, smem, st>>>(M, T, nwork);
  }
  return cudaGetLastError();
}

template <int TX, int TY, int TB, typename R>
static cudaError_t launch_tile(const MultiInst &M, cudaStream_t st) {
  return M.n == 1 ? launch_tile_n<TX, TY, TB, true, R>(M, st) : launch_tile_n<TX, TY, TB, false, R>(M, st);
}

int fast_tile_shapes(int *tx, int *ty, int *tg, int nmax) {
  static const int shapes[][3] = {{16, 16, 4}, {16, 16, 8}, {16, 16, 2}, {14, 14, 4}, {32, 8, 4}, {16, 12, 4}, {12, 16, 4},
                                  {16, 12, 8}};
  const int n = sizeof(shapes) / sizeof(shapes[0]);
  if (tx)
    for (int i = 0; i < n; ++i) tx[i] = shapes[i][0], ty[i] = shapes[i][1], tg[i] = shapes[i][2];
  (void)nmax;
  return n;
}

cudaError_t fast_build_offsets(const FastInst &I, float *off, cudaStream_t st) {
  const long long n = (long long)I.lall * I.gall;
  k_fast_offsets<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(I, off);
  return cudaGetLastError();
}
cudaError_t fast_build_offsets64(const FastInst &I, double *off, cudaStream_t st) {
  const long long n = (long long)I.lall * I.gall;
  k_fast_offsets<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(I, off);
  return cudaGetLastError();
}

cudaError_t fast_step_multi(const MultiInst &M, int shape, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                            long long &launches, unsigned parts) {
  if (M.n < 1 || M.n > kMaxInst) return cudaErrorInvalidValue;
  for (int i = 0; i < M.n; ++i)
    if (M.inst[i].l0 < 0 || M.inst[i].l1 > M.inst[i].lall || M.inst[i].l1 <= M.inst[i].l0) return cudaErrorInvalidValue;
  long long nbk = 0, nsk = 0, npl = 0, nc = 0, nvb = 0, nvb64 = 0, nfk = 0;
  int kmax = 0;
  constexpr int TV = 4, TV64 = 2;  // tracers per column thread: FP32, FP64 variant
  for (int i = 0; i < M.n; ++i) {
    const FastInst &I = M.inst[i];
    const long long n = I.gmax - I.gmin + 1, ncol = (long long)(I.l1 - I.l0) * n * n;
    nbk += (long long)I.nb * (I.K - 2);
    nsk += (long long)I.ns * (I.K - 2);
    nfk += (long long)(I.l1 - I.l0) * (I.K - 2) * I.gall;
    npl += I.poles ? (long long)kLallPl * I.ntr : 0LL;
    nc += (long long)I.ncarry * I.K;
    nvb += (long long)((I.ntr + TV - 1) / TV) * ((ncol + 255) / 256);
    nvb64 += (long long)((I.ntr + TV64 - 1) / TV64) * ((ncol + 255) / 256);
    kmax = I.K > kmax ? I.K : kmax;
  }
  if (kmax > 128) return cudaErrorInvalidValue;
  if (parts & 1u) {  // the boundary values other regions read (exchanged between ranks when sharded)
    k_fast_boundary<<<(unsigned)((nbk + 127) / 128), 128, 0, st>>>(M);
    launches += 1;
  }
  if (!(parts & 2u)) return cudaGetLastError();
  k_fast_seam<<<(unsigned)((nsk + 127) / 128), 128, 0, st>>>(M);
  if (npl > 0) {
    if (kmax <= 64) k_fast_pole<64><<<(unsigned)npl, 64, 0, st>>>(M);
    else k_fast_pole<128><<<(unsigned)npl, 128, 0, st>>>(M);
    launches += 1;
  }
  if (ev0) cudaEventRecord(ev0, st);
  const bool f64 = M.inst[0].f64 != 0;
  for (int i = 1; i < M.n; ++i)
    if ((M.inst[i].f64 != 0) != f64) return cudaErrorInvalidValue;  // one precision per batch
  cudaError_t e;
  if (!f64) {
    k_fast_faces<float><<<(unsigned)((nfk + 127) / 128), 128, 0, st>>>(M);
    switch (shape) {
      case 0: e = launch_tile<16, 16, 4, float>(M, st); break;
      case 1: e = launch_tile<16, 16, 8, float>(M, st); break;
      case 2: e = launch_tile<16, 16, 2, float>(M, st); break;
      case 3: e = launch_tile<14, 14, 4, float>(M, st); break;
      case 4: e = launch_tile<32, 8, 4, float>(M, st); break;
      case 5: e = launch_tile<16, 12, 4, float>(M, st); break;
      case 6: e = launch_tile<12, 16, 4, float>(M, st); break;
      case 7: e = launch_tile<16, 12, 8, float>(M, st); break;
      default: return cudaErrorInvalidValue;
    }
  } else {  // FP64 variant: the same tiles, 2 tracers per batch (FP64 shared data and registers)
    k_fast_faces<double><<<(unsigned)((nfk + 127) / 128), 128, 0, st>>>(M);
    switch (shape) {
      case 0: case 1: case 2: e = launch_tile<16, 16, 2, double>(M, st); break;
      case 3: e = launch_tile<14, 14, 2, double>(M, st); break;
      case 4: e = launch_tile<32, 8, 2, double>(M, st); break;
      case 5: e = launch_tile<16, 12, 2, double>(M, st); break;
      case 6: e = launch_tile<12, 16, 2, double>(M, st); break;
      case 7: e = launch_tile<16, 12, 2, double>(M, st); break;
      default: return cudaErrorInvalidValue;
    }
  }
  if (ev1) cudaEventRecord(ev1, st);
  if (e != cudaSuccess) return e;
  constexpr int vsm = (int)sizeof(VertRing<TV, float>), vsm64 = (int)sizeof(VertRing<TV64, double>);
  static_assert(vsm <= 48 * 1024 && vsm64 <= 48 * 1024, "the column ring fits the default shared-memory limit");
  if (!f64) {
    if (M.n == 1) k_fast_vert1<TV, float><<<(unsigned)nvb, 256, vsm, st>>>(M.inst[0]);
    else k_fast_vert<TV, float><<<(unsigned)nvb, 256, vsm, st>>>(M);
  } else {
    if (M.n == 1) k_fast_vert1<TV64, double><<<(unsigned)nvb64, 256, vsm64, st>>>(M.inst[0]);
    else k_fast_vert<TV64, double><<<(unsigned)nvb64, 256, vsm64, st>>>(M);
  }
  k_fast_carry<<<(unsigned)((nc + 127) / 128), 128, 0, st>>>(M);
  launches += 5;
  return cudaGetLastError();
}

cudaError_t fast_step(const FastInst &I, int shape, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                      long long &launches, unsigned parts) {
  MultiInst M;
  M.n = 1;
  M.inst[0] = I;
  return fast_step_multi(M, shape, st, ev0, ev1, launches, parts);
}

// ---- region-sharded runs: the exchanges' pack and unpack (contiguous buffers, no peer access)
__global__ void k_bval_copy(const int *bidx, int n, int nb, int K, int ntr, double *bbuf, double *buf, int unpack) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * K * ntr * 5) return;
  const int v = (int)(t % 5);
  long long r = t / 5;
  const int e = (int)(r % n);
  r /= n;  // = tr * K + k
  double *a = bbuf + ((size_t)r * nb + bidx[e]) * 5 + v;
  double *b = buf + ((size_t)r * n + e) * 5 + v;
  if (unpack) *a = *b;
  else *b = *a;
}
cudaError_t shard_bval_copy(const int *bidx, int n, int nb, int K, int ntr, double *bbuf, double *buf, bool unpack,
                            cudaStream_t st) {
  const long long total = (long long)n * K * ntr * 5;
  if (total == 0) return cudaSuccess;
  k_bval_copy<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(bidx, n, nb, K, ntr, bbuf, buf, unpack ? 1 : 0);
  return cudaGetLastError();
}
// points p of a (vmax, lall, kmax, gall) array and its (vmax, 2, kmax, 6) pole array <-> buf (vmax, kmax, n)
__global__ void k_point_copy(const int *pts, int n, int lall, int gall, int kmax, int vmax, double *var,
                             double *var_pl, double *buf, int unpack) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * kmax * vmax) return;
  const int e = (int)(t % n);
  const int k = (int)((t / n) % kmax), v = (int)(t / ((long long)n * kmax));
  const int p = pts[e];
  double *a;
  if (p < lall * gall) a = var + (((size_t)v * lall + p / gall) * kmax + k) * gall + p % gall;
  else {
    const int q = p - lall * gall;
    a = var_pl + (((size_t)v * kLallPl + q / kGallPl) * kmax + k) * kGallPl + q % kGallPl;
  }
  double *b = buf + ((size_t)v * kmax + k) * n + e;
  if (unpack) *a = *b;
  else *b = *a;
}
cudaError_t shard_point_copy(const int *pts, int n, int lall, int gall, int kmax, int vmax, double *var,
                             double *var_pl, double *buf, bool unpack, cudaStream_t st) {
  const long long total = (long long)n * kmax * vmax;
  if (total == 0) return cudaSuccess;
  k_point_copy<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(pts, n, lall, gall, kmax, vmax, var, var_pl, buf,
                                                                unpack ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace icoadv
