// Fused batched tracer step: FP32 flux-form remap / limiter arithmetic on
// interior faces, FP64 on region-seam faces, FP64 rhog / rhogq mass update.
//
// Per step, on the context stream:
//   k_fast_boundary  gradient and Thuburn outflow bounds Qout (FP64) of every
//                    region-boundary cell and both pole centres, into bbuf.  These
//                    are exactly the values the reference's two mid-step halo
//                    exchanges (grad q and Qout, mod_src_tracer.f90:371) would move
//                    into other regions' halos, so no exchange is needed.
//   k_fast_pole      the two pole centres (horizontal + vertical), FP64.
//   k_fast_tile      one CTA per (region tile, group of TG tracers), looping over the
//                    levels: fluxes (FP64, once per level), per tracer gradient,
//                    Qout, upwind remap and limiter (FP32), FP64 update, and the
//                    vertical sub-step streamed two levels behind in registers.
//   k_fast_carry     halo points that no halo list writes keep their input values.
//   gather           halo/pole fill of the new state (the COMM plan).
//
// Faces are "seam" faces when one of their two cells is a halo cell; the
// neighbouring region computes the same face from its own halo copy, so those
// faces are done in FP64 (k_fast_tile calls seam_face) to keep the flux form
// conservative to rounding of FP64.  Interior faces are computed by the same
// code in every tile that touches them, so they cancel exactly.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

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
    const float *p = var == 1 ? I->vx : (var == 2 ? I->vy : I->vz);
    return (double)p[off];
  }
};
struct GQ {
  const FastInst *I;
  int l, k, t;
  __device__ double operator()(int i, int j) const {
    const size_t off = ((size_t)l * I->K + k) * I->gall + (size_t)(j - 1) * I->G + (i - 1);
    return I->Q_in[(size_t)t * I->lall * I->K * I->gall + off] / I->rho_in[off];
  }
};

// ---- poles: the 5 ring faces of pole p at level k (mod_src_tracer.f90:326-374), FP64
__device__ void pole_faces(const FastInst &I, int p, int k, double flux[7], double xc[7][3]) {
  const size_t off = ((size_t)p * I.K + k) * kGallPl;
  auto GT = [&](int v, int w) { return I.GMTR_t_pl[((size_t)(w - 1) * kLallPl + p) * kGallPl + (v - 1)]; };
  auto GA = [&](int v, int h) { return I.GMTR_a_pl[((size_t)(h - 1) * kLallPl + p) * kGallPl + (v - 1)]; };
  auto R = [&](int v) { return I.rho_in_pl[off + v - 1]; };
  auto X = [&](int v) { return (double)I.vx_pl[off + v - 1]; };
  auto Y = [&](int v) { return (double)I.vy_pl[off + v - 1]; };
  auto Z = [&](int v) { return (double)I.vz_pl[off + v - 1]; };
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

// Qout of pole centre p at level k for tracer t (mod_src_tracer.f90:307-363), d = 0
__device__ void pole_qout(const FastInst &I, int p, int k, int t, const double flux[7], double &Qmin, double &Qmax) {
  const size_t off = ((size_t)p * I.K + k) * kGallPl;
  const size_t toff = (size_t)t * kLallPl * I.K * kGallPl;
  double q[7];
  for (int v = 1; v <= 6; ++v) q[v] = I.Q_in_pl[toff + off + v - 1] / I.rho_in_pl[off + v - 1];
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

// ---- FP64 gradient and Qout of an interior region cell (i,j) (boundary pass)
__device__ void cell_grad_qout64(const FastInst &I, int l, int k, int t, int i, int j, double out[5]) {
  const bool sgp = I.have_sgp[l] != 0;
  const GFields f{&I, l, k};
  const GQ q{&I, l, k, t};
  const int G = I.G, c = (j - 1) * G + (i - 1);
  // gradient (stencil of OPRT_gradient_setup), neighbour order ij, ip1j, ip1jp1, ijp1, im1j, im1jm1, ijm1
  const int di[7] = {0, 1, 1, 0, -1, -1, 0}, dj[7] = {0, 0, 1, 1, 0, -1, -1};
  double qs[7];
  for (int n = 0; n < 7; ++n) qs[n] = q(i + di[n], j + dj[n]);
  for (int x = 0; x < 3; ++x) {
    const double *cx = I.cg + ((size_t)l * 3 + x) * 7 * I.gall + c;
    double s = cx[0] * qs[0];
    for (int n = 1; n <= 6; ++n) s = s + cx[(size_t)n * I.gall] * qs[n];
    out[x] = s;
  }
  // Qout (mod_src_tracer.f90:143-282) with d = 0
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  const int oi[7] = {0, i, i, i, i - 1, i - 1, i}, oj[7] = {0, j, j, j, j, j - 1, j - 1};
  const int fa[7] = {0, AI, AIJ, AJ, AI, AIJ, AJ};
  const double rho_c = f(0, i, j), ra_c = rarea(I, l, i, j);
  double qmn[7], qmx[7], ch[7], chm[7];
  for (int m = 1; m <= 6; ++m) {
    double xc[3];
    const bool ex = face_exists(I, oi[m], oj[m], fa[m]);
    const double fl = ex ? face_geo(I, l, oi[m], oj[m], fa[m], sgp, f, xc) : 0.0;
    const double flx = ex ? cell_flx(I, l, i, j, m, sgp, fl, ra_c) : 0.0;
    ch[m] = flx / rho_c;
    chm[m] = mn64(ch[m], 0.0);
    // upwind mask of the face, from its owner's Courant number
    const double ch_own = (m <= 3) ? ch[m] : (fl * rarea(I, l, oi[m], oj[m]) * I.dt) / f(0, oi[m], oj[m]);
    const double cm = 0.5 - fsg(0.5, ch_own - EPS);
    double lo, hi;
    bounds64(I, oi[m], oj[m], fa[m], sgp, q, lo, hi);
    if (m <= 3) qmn[m] = cm * lo + (1.0 - cm) * BIG, qmx[m] = cm * hi + (1.0 - cm) * (-BIG);
    else qmn[m] = cm * BIG + (1.0 - cm) * lo, qmx[m] = cm * (-BIG) + (1.0 - cm) * hi;
  }
  const double q0 = qs[0];
  double qnmin = q0, qnmax = q0;
  for (int m = 1; m <= 6; ++m) qnmin = mn64(qnmin, qmn[m]);
  for (int m = 1; m <= 6; ++m) qnmax = mx64(qnmax, qmx[m]);
  const double Cin = chm[1] + chm[2] + chm[3] + chm[4] + chm[5] + chm[6];
  const double Cout =
      ch[1] - chm[1] + ch[2] - chm[2] + ch[3] - chm[3] + ch[4] - chm[4] + ch[5] - chm[5] + ch[6] - chm[6];
  const double CQmin = chm[1] * qmn[1] + chm[2] * qmn[2] + chm[3] * qmn[3] + chm[4] * qmn[4] + chm[5] * qmn[5] +
                       chm[6] * qmn[6];
  const double CQmax = chm[1] * qmx[1] + chm[2] * qmx[2] + chm[3] * qmx[3] + chm[4] * qmx[4] + chm[5] * qmx[5] +
                       chm[6] * qmx[6];
  const double zerosw = 0.5 - fsg(0.5, fabs(Cout) - EPS);
  out[3] = (q0 - CQmax - qnmax * (1.0 - Cin - Cout + 0.0)) / (Cout + zerosw) * (1.0 - zerosw) + q0 * zerosw;
  out[4] = (q0 - CQmin - qnmin * (1.0 - Cin - Cout + 0.0)) / (Cout + zerosw) * (1.0 - zerosw) + q0 * zerosw;
}

__global__ void k_fast_boundary(FastInst I) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)I.nb * (I.K - 2) * I.ntr;
  if (tid >= total) return;
  const int b = (int)(tid % I.nb);
  const long long r = tid / I.nb;
  const int k = 1 + (int)(r % (I.K - 2)), t = (int)(r / (I.K - 2));
  double out[5];
  const int p = I.blist[b];
  if (p < I.lall * I.gall) {
    const int l = p / I.gall, c = p % I.gall;
    cell_grad_qout64(I, l, k, t, c % I.G + 1, c / I.G + 1, out);
  } else {  // pole centre
    const int pl = (p - I.lall * I.gall) / kGallPl;
    const size_t off = ((size_t)pl * I.K + k) * kGallPl;
    const size_t toff = (size_t)t * kLallPl * I.K * kGallPl;
    double q[7];
    for (int v = 1; v <= 6; ++v) q[v] = I.Q_in_pl[toff + off + v - 1] / I.rho_in_pl[off + v - 1];
    for (int x = 0; x < 3; ++x) {
      const double *cx = I.cg_pl + ((size_t)pl * 3 + x) * 6;
      double s = cx[0] * q[1];
      for (int v = 2; v <= 6; ++v) s = s + cx[v - 1] * q[v];
      out[x] = s;
    }
    double flux[7], xc[7][3];
    pole_faces(I, pl, k, flux, xc);
    pole_qout(I, pl, k, t, flux, out[3], out[4]);
  }
  double *dst = I.bbuf + (((size_t)t * I.K + k) * I.nb + b) * 5;
  for (int x = 0; x < 5; ++x) dst[x] = out[x];
}

__device__ __forceinline__ const double *bval(const FastInst &I, int t, int k, int b) {
  return I.bbuf + (((size_t)t * I.K + k) * I.nb + b) * 5;
}

// ---- the value of a seam face (one side a halo cell), FP64, from global memory
__device__ double seam_face(const FastInst &I, int l, int k, int t, int i, int j, int a, double flux,
                            const double xc[3]) {
  const bool sgp = I.have_sgp[l] != 0;
  const GFields f{&I, l, k};
  const GQ q{&I, l, k, t};
  const int G = I.G;
  const int ni = (a == AI || a == AIJ) ? i + 1 : i, nj = (a == AIJ || a == AJ) ? j + 1 : j;
  const double ch = (flux * rarea(I, l, i, j) * I.dt) / f(0, i, j);
  const double cm = 0.5 - fsg(0.5, ch - DBL_EPSILON);
  const int bo = I.bsrc[(size_t)l * I.gall + (j - 1) * G + (i - 1)];
  const int bn = I.bsrc[(size_t)l * I.gall + (nj - 1) * G + (ni - 1)];
  // gradient and Qout of both cells (both are boundary or halo cells of this region)
  double go[5] = {0, 0, 0, 0, 0}, gn[5] = {0, 0, 0, 0, 0};
  const double qo = q(i, j), qn = q(ni, nj);
  if (bo >= 0) for (int x = 0; x < 5; ++x) go[x] = bval(I, t, k, bo)[x];
  else go[3] = go[4] = qo;  // halo point no list reaches: Qout = q, grad = 0 (as after the reference fill)
  if (bn >= 0) for (int x = 0; x < 5; ++x) gn[x] = bval(I, t, k, bn)[x];
  else gn[3] = gn[4] = qn;
  double vu = qn, vs = qo;
  for (int x = 0; x < 3; ++x) vu = vu + gn[x] * (xc[x] - gx(I, l, ni, nj, x));
  for (int x = 0; x < 3; ++x) vs = vs + go[x] * (xc[x] - gx(I, l, i, j, x));
  double v = cm * vu + (1.0 - cm) * vs;
  double lo, hi;
  bounds64(I, i, j, a, sgp, q, lo, hi);
  const double BIG = DBL_MAX;
  const double own_min = cm * lo + (1.0 - cm) * BIG, own_max = cm * hi + (1.0 - cm) * (-BIG);
  const double nb_min = cm * BIG + (1.0 - cm) * lo, nb_max = cm * (-BIG) + (1.0 - cm) * hi;
  v = cm * mn64(mx64(v, own_min), own_max) + (1.0 - cm) * mn64(mx64(v, nb_min), nb_max);
  v = cm * mx64(mn64(v, gn[4]), gn[3]) + (1.0 - cm) * mx64(mn64(v, go[4]), go[3]);
  return v;
}

// ---- the fused tile kernel ----------------------------------------------------------
// local frame: region coords (i,j) -> local (i - i0 + 3, j - j0 + 3), size (TX+5) x (TY+5)
template <int TX, int TY>
struct TileSmem {
  static constexpr int W = TX + 5, H = TY + 5, N = W * H;
  double rho[N];
  double flux[3][N];
  double qa[3][N];
  float v[3][N];
  float xc[3][3][N];
  float cm[3][N];
  float q[N];
  float gq[5][N];
};

template <int TX, int TY, int TG>
__global__ void __launch_bounds__(TX *TY) k_fast_tile(FastInst I) {
  using S = TileSmem<TX, TY>;
  constexpr int W = S::W, N = S::N, NT = TX * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);

  const int ngroups = (I.ntr + TG - 1) / TG;
  const int grp = blockIdx.x % ngroups;
  const int tile = blockIdx.x / ngroups;
  const int tiles_per_rgn = I.ntx * I.nty;
  const int l = tile / tiles_per_rgn;
  const int tr = tile % tiles_per_rgn;
  const int i0 = I.gmin + (tr % I.ntx) * TX, j0 = I.gmin + (tr / I.ntx) * TY;
  const int t0 = grp * TG;
  const int ntg = min(TG, I.ntr - t0);
  const int tid = threadIdx.x;
  const int ti = tid % TX, tj = tid / TX;
  const int ci = i0 + ti, cj = j0 + tj;  // this thread's cell
  const bool active = ci <= I.gmax && cj <= I.gmax;
  const bool sgp = I.have_sgp[l] != 0;
  const int G = I.G, K = I.K;
  const size_t slab = (size_t)I.gall, lk = (size_t)K * I.gall, tstride = (size_t)I.lall * K * I.gall;
  const double dt = I.dt;
  const double ra_c = active ? rarea(I, l, ci, cj) : 1.0;
  const size_t ccell = (size_t)(cj - 1) * G + (ci - 1);
  auto LI = [&](int i, int j) { return (j - j0 + 3) * W + (i - i0 + 3); };
  auto inreg = [&](int i, int j) { return i >= 1 && i <= G && j >= 1 && j <= G; };
  auto interior = [&](int i, int j) { return i >= I.gmin && i <= I.gmax && j >= I.gmin && j <= I.gmax; };

  // vertical window, per tracer of the group (registers)
  double Qh[TG][3];
  float qv[TG][3], qmn_km1[TG], qmx_km1[TG], qh_last[TG];
  double rh[3];    // rho after the horizontal sub-step at levels k-2, k-1, k
  float ck1w[3];   // ck(k,1) at levels k-2..k
  float ck2w[3];
  float wf[3];     // rhogw at faces k-2..k (face k = below level k)
  double rnew_prev = 0.0;
  (void)rnew_prev;

  const float BIGf = FLT_MAX, EPSf = FLT_EPSILON;

  // vertical Qout of level slot `mid` (window index 1 = level L) using q at L-1, L, L+1 (FP32)
  auto vqout32 = [&](float qm, float qk, float qp, float c1, float c2, float c1p, float &infl, float &Qmin,
                     float &Qmax) {
    infl = 0.5f - copysignf(0.5f, c1);
    const float infu = 0.5f + copysignf(0.5f, c1p);
    const float minL = mn32(qk, qm) + (1.0f - infl) * BIGf;
    const float minU = mn32(qk, qp) + (1.0f - infu) * BIGf;
    const float maxL = mx32(qk, qm) - (1.0f - infl) * BIGf;
    const float maxU = mx32(qk, qp) - (1.0f - infu) * BIGf;
    const float qnmin = mn32(mn32(minL, minU), qk);
    const float qnmax = mx32(mx32(maxL, maxU), qk);
    const float Cin = infl * c1 + infu * c2;
    const float Cout = (1.0f - infl) * c1 + (1.0f - infu) * c2;
    const float CQmin = infl * c1 * minL + infu * c2 * minU;
    const float CQmax = infl * c1 * maxL + infu * c2 * maxU;
    const float zerosw = 0.5f - copysignf(0.5f, fabsf(Cout) - EPSf);
    Qmin = ((qk - qnmax) + qnmax * (Cin + Cout) - CQmax) / (Cout + zerosw) * (1.0f - zerosw) + qk * zerosw;
    Qmax = ((qk - qnmin) + qnmin * (Cin + Cout) - CQmin) / (Cout + zerosw) * (1.0f - zerosw) + qk * zerosw;
  };

  // write one finished level of one tracer
  auto store = [&](int tt, int L, double val) {
    if (!active) return;
    I.Q_out[(size_t)(t0 + tt) * tstride + (size_t)l * lk + (size_t)L * slab + ccell] = val;
  };

  for (int k = 1; k <= K - 2; ++k) {
    // ---- (1) shared fields of this level in the tile window
    const size_t base = (size_t)l * lk + (size_t)k * slab;
    for (int e = tid; e < N; e += NT) {
      const int i = i0 - 3 + e % W, j = j0 - 3 + e / W;
      if (inreg(i, j)) {
        const size_t o = base + (size_t)(j - 1) * G + (i - 1);
        s.rho[e] = I.rho_in[o];
        s.v[0][e] = I.vx[o];
        s.v[1][e] = I.vy[o];
        s.v[2][e] = I.vz[o];
      } else {
        s.rho[e] = 1.0;
        s.v[0][e] = s.v[1][e] = s.v[2][e] = 0.0f;
      }
    }
    __syncthreads();
    // ---- (2) faces of owners in [-2, T]^2 (local 1..T+3): FP64 flux, FP32 centroid, upwind mask
    {
      auto acc = [&](int var, int i, int j) -> double {
        const int e = LI(i, j);
        return var == 0 ? s.rho[e] : (double)s.v[var - 1][e];
      };
      for (int e = tid; e < N; e += NT) {
        const int lx = e % W, ly = e / W;
        const int i = i0 - 3 + lx, j = j0 - 3 + ly;
        const bool own = lx >= 1 && ly >= 1 && lx <= TX + 3 && ly <= TY + 3 && i >= 1 && j >= 1 && i < G && j < G;
        for (int a = 1; a <= 3; ++a) {
          double fl = 0.0, xc[3] = {0, 0, 0};
          if (own && face_exists(I, i, j, a)) fl = face_geo(I, l, i, j, a, sgp, acc, xc);
          s.flux[a - 1][e] = fl;
          s.xc[0][a - 1][e] = (float)xc[0];
          s.xc[1][a - 1][e] = (float)xc[1];
          s.xc[2][a - 1][e] = (float)xc[2];
          double cmv = 1.0;
          if (own && inreg(i, j)) {
            const double chv = (fl * rarea(I, l, i, j) * dt) / s.rho[e];
            cmv = 0.5 - fsg(0.5, chv - DBL_EPSILON);
          }
          s.cm[a - 1][e] = (float)cmv;
        }
      }
    }
    __syncthreads();
    // ---- per-thread fluxes of its cell (FP64) and the density after the horizontal sub-step
    double flx[7];
    double rho_h = 0.0;
    if (active) {
      const int e = LI(ci, cj);
      flx[1] = cell_flx(I, l, ci, cj, 1, sgp, s.flux[0][e], ra_c);
      flx[2] = cell_flx(I, l, ci, cj, 2, sgp, s.flux[1][e], ra_c);
      flx[3] = cell_flx(I, l, ci, cj, 3, sgp, s.flux[2][e], ra_c);
      flx[4] = cell_flx(I, l, ci, cj, 4, sgp, s.flux[0][e - 1], ra_c);
      flx[5] = cell_flx(I, l, ci, cj, 5, sgp, s.flux[1][e - W - 1], ra_c);
      flx[6] = cell_flx(I, l, ci, cj, 6, sgp, s.flux[2][e - W], ra_c);
      double sum = flx[1];
      for (int m = 2; m <= 6; ++m) sum = sum + flx[m];
      rho_h = s.rho[e] - sum;
    }
    // vertical window of shared quantities (slot 2 = level k)
    rh[0] = rh[1];
    rh[1] = rh[2];
    rh[2] = rho_h;
    wf[0] = wf[1];
    wf[1] = wf[2];
    wf[2] = active ? I.w[base + ccell] : 0.0f;
    const float wtop = active ? I.w[base + slab + ccell] : 0.0f;  // face k+1
    ck1w[0] = ck1w[1];
    ck1w[1] = ck1w[2];
    ck2w[0] = ck2w[1];
    ck2w[1] = ck2w[2];
    ck1w[2] = (float)(-(double)wf[2] * dt * I.rdgz[k] / rho_h);
    ck2w[2] = (float)((double)wtop * dt * I.rdgz[k] / rho_h);

#pragma unroll
    for (int tt = 0; tt < TG; ++tt) {
      if (tt >= ntg) break;
      const int t = t0 + tt;
      const double *Qt = I.Q_in + (size_t)t * tstride + base;
      // ---- (a) q in the window (FP32)
      for (int e = tid; e < N; e += NT) {
        const int i = i0 - 3 + e % W, j = j0 - 3 + e / W;
        s.q[e] = inreg(i, j) ? (float)(Qt[(size_t)(j - 1) * G + (i - 1)] / s.rho[e]) : 0.0f;
      }
      __syncthreads();
      // ---- (b) gradient and Qout of cells in [-1, T]^2
      for (int e = tid; e < N; e += NT) {
        const int lx = e % W, ly = e / W;
        if (lx < 2 || ly < 2 || lx > TX + 3 || ly > TY + 3) continue;
        const int i = i0 - 3 + lx, j = j0 - 3 + ly;
        if (!inreg(i, j)) continue;
        const int bs = I.bsrc[(size_t)l * I.gall + (j - 1) * G + (i - 1)];
        if (bs >= 0) {
          const double *bv = bval(I, t, k, bs);
          for (int x = 0; x < 5; ++x) s.gq[x][e] = (float)bv[x];
          continue;
        }
        if (bs == -2) {
          s.gq[0][e] = s.gq[1][e] = s.gq[2][e] = 0.0f;
          s.gq[3][e] = s.gq[4][e] = s.q[e];
          continue;
        }
        // interior cell one or more cells away from the region edge: FP32
        const int c = (j - 1) * G + (i - 1);
        const int nbe[7] = {e, e + 1, e + W + 1, e + W, e - 1, e - W - 1, e - W};
        for (int x = 0; x < 3; ++x) {
          const float *cx = I.cg32 + ((size_t)l * 3 + x) * 7 * I.gall + c;
          float g = __ldg(cx) * s.q[nbe[0]];
          for (int n = 1; n <= 6; ++n) g = g + __ldg(cx + (size_t)n * I.gall) * s.q[nbe[n]];
          s.gq[x][e] = g;
        }
        const float q0 = s.q[e];
        const float rhoc = (float)s.rho[e];
        const float rac = (float)rarea(I, l, i, j);
        // the 6 faces: owner slot and face type
        const int oe[7] = {0, e, e, e, e - 1, e - W - 1, e - W};
        const int fa[7] = {0, 0, 1, 2, 0, 1, 2};
        float qmn[7], qmx[7], ch[7], chm[7];
#pragma unroll
        for (int m = 1; m <= 6; ++m) {
          const int o = oe[m];
          const float fl = (float)s.flux[fa[m]][o];
          const float flxm = (m <= 3 ? fl : -fl) * rac * (float)dt;
          ch[m] = flxm / rhoc;
          chm[m] = mn32(ch[m], 0.0f);
          const float cm = s.cm[fa[m]][o];
          // 4-point bounds of the face around its owner o
          float b1, b2, b3;
          const float qo = s.q[o];
          if (fa[m] == 0) b1 = s.q[o - W], b2 = s.q[o + 1], b3 = s.q[o + W + 1];
          else if (fa[m] == 1) b1 = s.q[o + 1], b2 = s.q[o + W + 1], b3 = s.q[o + W];
          else b1 = s.q[o + W + 1], b2 = s.q[o + W], b3 = s.q[o - 1];
          const float lo = mn32(mn32(mn32(qo, b1), b2), b3), hi = mx32(mx32(mx32(qo, b1), b2), b3);
          if (m <= 3) qmn[m] = cm * lo + (1.0f - cm) * BIGf, qmx[m] = cm * hi + (1.0f - cm) * (-BIGf);
          else qmn[m] = cm * BIGf + (1.0f - cm) * lo, qmx[m] = cm * (-BIGf) + (1.0f - cm) * hi;
        }
        float qnmin = q0, qnmax = q0;
#pragma unroll
        for (int m = 1; m <= 6; ++m) qnmin = mn32(qnmin, qmn[m]), qnmax = mx32(qnmax, qmx[m]);
        const float Cin = chm[1] + chm[2] + chm[3] + chm[4] + chm[5] + chm[6];
        const float Cout =
            ch[1] - chm[1] + ch[2] - chm[2] + ch[3] - chm[3] + ch[4] - chm[4] + ch[5] - chm[5] + ch[6] - chm[6];
        const float CQmin = chm[1] * qmn[1] + chm[2] * qmn[2] + chm[3] * qmn[3] + chm[4] * qmn[4] +
                            chm[5] * qmn[5] + chm[6] * qmn[6];
        const float CQmax = chm[1] * qmx[1] + chm[2] * qmx[2] + chm[3] * qmx[3] + chm[4] * qmx[4] +
                            chm[5] * qmx[5] + chm[6] * qmx[6];
        const float zerosw = 0.5f - copysignf(0.5f, fabsf(Cout) - EPSf);
        s.gq[3][e] = (q0 - CQmax - qnmax * (1.0f - Cin - Cout)) / (Cout + zerosw) * (1.0f - zerosw) + q0 * zerosw;
        s.gq[4][e] = (q0 - CQmin - qnmin * (1.0f - Cin - Cout)) / (Cout + zerosw) * (1.0f - zerosw) + q0 * zerosw;
      }
      __syncthreads();
      // ---- (c) limited face values of owners in [-1, T-1]^2
      for (int e = tid; e < N; e += NT) {
        const int lx = e % W, ly = e / W;
        if (lx < 2 || ly < 2 || lx > TX + 2 || ly > TY + 2) continue;
        const int i = i0 - 3 + lx, j = j0 - 3 + ly;
        if (!inreg(i, j)) continue;
        const int nbe[3] = {e + 1, e + W + 1, e + W};
        const int nbi[3] = {i + 1, i + 1, i}, nbj[3] = {j, j + 1, j + 1};
        const bool own_in = interior(i, j);
        for (int a = 0; a < 3; ++a) {
          if (!face_exists(I, i, j, a + 1)) {
            s.qa[a][e] = 0.0;
            continue;
          }
          const int n = nbe[a];
          if (!own_in || !interior(nbi[a], nbj[a])) {  // seam face: FP64 from global memory
            double xc[3];
            const GFields f{&I, l, k};
            const double fl = face_geo(I, l, i, j, a + 1, sgp, f, xc);
            s.qa[a][e] = seam_face(I, l, k, t, i, j, a + 1, fl, xc);
            continue;
          }
          const float cm = s.cm[a][e];
          float vu = s.q[n], vs = s.q[e];
          for (int x = 0; x < 3; ++x) {
            const float xcv = s.xc[x][a][e];
            vu = vu + s.gq[x][n] * (xcv - (float)gx(I, l, nbi[a], nbj[a], x));
          }
          for (int x = 0; x < 3; ++x) {
            const float xcv = s.xc[x][a][e];
            vs = vs + s.gq[x][e] * (xcv - (float)gx(I, l, i, j, x));
          }
          float v = cm * vu + (1.0f - cm) * vs;
          float b1, b2, b3;
          const float qo = s.q[e];
          if (a == 0) b1 = s.q[e - W], b2 = s.q[e + 1], b3 = s.q[e + W + 1];
          else if (a == 1) b1 = s.q[e + 1], b2 = s.q[e + W + 1], b3 = s.q[e + W];
          else b1 = s.q[e + W + 1], b2 = s.q[e + W], b3 = s.q[e - 1];
          const float lo = mn32(mn32(mn32(qo, b1), b2), b3), hi = mx32(mx32(mx32(qo, b1), b2), b3);
          const float own_min = cm * lo + (1.0f - cm) * BIGf, own_max = cm * hi + (1.0f - cm) * (-BIGf);
          const float nb_min = cm * BIGf + (1.0f - cm) * lo, nb_max = cm * (-BIGf) + (1.0f - cm) * hi;
          v = cm * mn32(mx32(v, own_min), own_max) + (1.0f - cm) * mn32(mx32(v, nb_min), nb_max);
          v = cm * mx32(mn32(v, s.gq[4][n]), s.gq[3][n]) + (1.0f - cm) * mx32(mn32(v, s.gq[4][e]), s.gq[3][e]);
          s.qa[a][e] = (double)v;
        }
      }
      __syncthreads();
      // ---- (d) horizontal update of this thread's cell (FP64) and (e) the vertical stream
      if (active) {
        const int e = LI(ci, cj);
        const double qa[7] = {0, s.qa[0][e], s.qa[1][e], s.qa[2][e], s.qa[0][e - 1], s.qa[1][e - W - 1],
                              s.qa[2][e - W]};
        double sum = flx[1] * qa[1];
        for (int m = 2; m <= 6; ++m) sum = sum + flx[m] * qa[m];
        const double Qhk = Qt[ccell] - sum;
        Qh[tt][0] = Qh[tt][1];
        Qh[tt][1] = Qh[tt][2];
        Qh[tt][2] = Qhk;
        qv[tt][0] = qv[tt][1];
        qv[tt][1] = qv[tt][2];
        qv[tt][2] = (float)(Qhk / rho_h);
        if (k == 1) {  // ghost level below: q(kmin-1) = q(kmin)
          qv[tt][1] = qv[tt][2];
          qh_last[tt] = 0.0f;
        }
        if (k >= 2) {
          // Qout of level k-1 (window slot 1) from q at k-2, k-1, k
          float infl, Qmin, Qmax;
          vqout32(qv[tt][0], qv[tt][1], qv[tt][2], ck1w[1], ck2w[1], ck1w[2], infl, Qmin, Qmax);
          // face k-1 (between levels k-2 and k-1)
          const int f = k - 1;
          float qh = (float)I.afact[f] * qv[tt][1] + (float)I.bfact[f] * qv[tt][0];
          if (f >= 2) {
            qh = infl * mx32(mn32(qh, qmx_km1[tt]), qmn_km1[tt]) + (1.0f - infl) * mx32(mn32(qh, Qmax), Qmin);
          }
          // level k-2 is final once faces k-2 and k-1 are
          if (k - 2 >= 1) {
            const int L = k - 2;
            const double fu = (double)wf[1] * (double)qh, fl = (double)wf[0] * (double)qh_last[tt];
            const double Qn = Qh[tt][0] - (fu - fl) * dt * I.rdgz[L];
            store(tt, L, Qn);
            if (L == 1) store(tt, 0, Qn);
          }
          qh_last[tt] = qh;
          qmn_km1[tt] = Qmin;
          qmx_km1[tt] = Qmax;
        }
      }
      __syncthreads();
    }
    // density: level k-2 final (one group writes it)
    if (active && grp == 0 && k >= 3) {
      const int L = k - 2;
      const double rn = rh[0] - ((double)wf[1] - (double)wf[0]) * dt * I.rdgz[L];
      I.rho_out[(size_t)l * lk + (size_t)L * slab + ccell] = rn;
      if (L == 1) I.rho_out[(size_t)l * lk + ccell] = rn;
    }
  }
  // ---- drain: levels K-3 and K-2 (faces K-2 and K-1)
  if (active) {
    const int kk = K - 1;  // ghost level above: q(kmax+1) = q(kmax)
    const float wtop = 0.0f;
    (void)wtop;
#pragma unroll
    for (int tt = 0; tt < TG; ++tt) {
      if (tt >= ntg) break;
      // Qout of level K-2 with q(K-1) := q(K-2)
      float infl, Qmin, Qmax;
      const float c1top = (float)(-(double)I.w[(size_t)l * lk + (size_t)kk * slab + ccell] * dt * I.rdgz[kk] /
                                  I.rho_in[(size_t)l * lk + (size_t)kk * slab + ccell]);
      vqout32(qv[tt][1], qv[tt][2], qv[tt][2], ck1w[2], ck2w[2], c1top, infl, Qmin, Qmax);
      const int f = K - 2;
      float qh = (float)I.afact[f] * qv[tt][2] + (float)I.bfact[f] * qv[tt][1];
      if (f >= 2) qh = infl * mx32(mn32(qh, qmx_km1[tt]), qmn_km1[tt]) + (1.0f - infl) * mx32(mn32(qh, Qmax), Qmin);
      if (K - 3 >= 1) {
        const int L = K - 3;
        const double fu = (double)wf[2] * (double)qh, fl = (double)wf[1] * (double)qh_last[tt];
        const double Qn = Qh[tt][1] - (fu - fl) * dt * I.rdgz[L];
        store(tt, L, Qn);
        if (L == 1) store(tt, 0, Qn);
      }
      // top face K-1: unlimited, rhogw = 0 there
      const float qtop = (float)I.afact[kk] * qv[tt][2] + (float)I.bfact[kk] * qv[tt][2];
      const float wk1 = I.w[(size_t)l * lk + (size_t)kk * slab + ccell];
      const double fu = (double)wk1 * (double)qtop, fl = (double)wf[2] * (double)qh;
      const double Qn = Qh[tt][2] - (fu - fl) * dt * I.rdgz[K - 2];
      store(tt, K - 2, Qn);
      store(tt, K - 1, Qn);
      if (K - 2 == 1) store(tt, 0, Qn);
    }
    if (grp == 0) {
      const float wk1 = I.w[(size_t)l * lk + (size_t)kk * slab + ccell];
      if (K - 3 >= 1) {
        const int L = K - 3;
        const double rn = rh[1] - ((double)wf[2] - (double)wf[1]) * dt * I.rdgz[L];
        I.rho_out[(size_t)l * lk + (size_t)L * slab + ccell] = rn;
        if (L == 1) I.rho_out[(size_t)l * lk + ccell] = rn;
      }
      const double rn = rh[2] - ((double)wk1 - (double)wf[2]) * dt * I.rdgz[K - 2];
      I.rho_out[(size_t)l * lk + (size_t)(K - 2) * slab + ccell] = rn;
      I.rho_out[(size_t)l * lk + (size_t)(K - 1) * slab + ccell] = rn;
      if (K - 2 == 1) I.rho_out[(size_t)l * lk + ccell] = rn;
    }
  }
}

// ---- the two pole centres, all levels, one thread per (pole, tracer), FP64 -----------
template <int KMAX>
__global__ void k_fast_pole(FastInst I) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kLallPl * I.ntr) return;
  const int p = t % kLallPl, tr = t / kLallPl;
  const int K = I.K;
  const size_t toff = (size_t)tr * kLallPl * K * kGallPl;
  const double rarea = I.GMTR_p_pl[((size_t)(P_RAREA - 1) * kLallPl + p) * kGallPl];
  double Qh[KMAX], rh[KMAX];
  for (int k = 1; k <= K - 2; ++k) {
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
    const double BIG = DBL_MAX, EPS = DBL_EPSILON;
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
    Qh[k] = I.Q_in_pl[toff + off] - sum;
    rh[k] = I.rho_in_pl[off] - rsum;
  }
  // vertical sub-step of the pole column (FP64, as the plain path)
  const int kmin = 1, kmax = K - 2;
  double ck1[KMAX], ck2[KMAX], q[KMAX], qh[KMAX];
  auto W = [&](int k) { return (double)I.w_pl[((size_t)p * K + k) * kGallPl]; };
  for (int k = 0; k < K; ++k) ck1[k] = ck2[k] = 0.0;
  for (int k = kmin; k <= kmax; ++k) {
    ck1[k] = -W(k) * I.dt * I.rdgz[k] / rh[k];
    ck2[k] = W(k + 1) * I.dt * I.rdgz[k] / rh[k];
  }
  ck1[K - 1] = -W(K - 1) * I.dt * I.rdgz[K - 1] / I.rho_in_pl[((size_t)p * K + K - 1) * kGallPl];
  for (int k = kmin; k <= kmax; ++k) q[k] = Qh[k] / rh[k];
  q[0] = q[kmin];
  q[K - 1] = q[kmax];
  for (int k = kmin; k <= kmax + 1 && k < K; ++k) qh[k] = I.afact[k] * q[k] + I.bfact[k] * q[k - 1];
  const double BIG = DBL_MAX, EPS = DBL_EPSILON;
  auto vq = [&](int k, double &infl, double &Qmin, double &Qmax) {
    infl = 0.5 - fsg(0.5, ck1[k]);
    const double infu = 0.5 + fsg(0.5, ck1[k + 1]);
    const double qk = q[k], qm = q[k - 1], qp = q[k + 1];
    const double minL = mn64(qk, qm) + (1.0 - infl) * BIG, minU = mn64(qk, qp) + (1.0 - infu) * BIG;
    const double maxL = mx64(qk, qm) - (1.0 - infl) * BIG, maxU = mx64(qk, qp) - (1.0 - infu) * BIG;
    const double qnmin = mn64(mn64(minL, minU), qk), qnmax = mx64(mx64(maxL, maxU), qk);
    const double Cin = infl * ck1[k] + infu * ck2[k], Cout = (1.0 - infl) * ck1[k] + (1.0 - infu) * ck2[k];
    const double CQmax = infl * ck1[k] * maxL + infu * ck2[k] * maxU;  // region form, as the composed step
    const double CQmin = infl * ck1[k] * minL + infu * ck2[k] * minU;
    const double zerosw = 0.5 - fsg(0.5, fabs(Cout) - EPS);
    Qmin = ((qk - qnmax) + qnmax * (Cin + Cout) - CQmax) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
    Qmax = ((qk - qnmin) + qnmin * (Cin + Cout) - CQmin) / (Cout + zerosw) * (1.0 - zerosw) + qk * zerosw;
  };
  double fl0, Qmin_km1, Qmax_km1;
  vq(kmin, fl0, Qmin_km1, Qmax_km1);
  for (int k = kmin + 1; k <= kmax; ++k) {
    double infl, Qmin, Qmax;
    vq(k, infl, Qmin, Qmax);
    const double h = qh[k];
    qh[k] = infl * mx64(mn64(h, Qmax_km1), Qmin_km1) + (1.0 - infl) * mx64(mn64(h, Qmax), Qmin);
    Qmin_km1 = Qmin, Qmax_km1 = Qmax;
  }
  for (int k = kmin; k <= kmax; ++k) {
    const double Qn = Qh[k] - (W(k + 1) * qh[k + 1] - W(k) * qh[k]) * I.dt * I.rdgz[k];
    I.Q_out_pl[toff + ((size_t)p * K + k) * kGallPl] = Qn;
  }
  I.Q_out_pl[toff + ((size_t)p * K + 0) * kGallPl] = I.Q_out_pl[toff + ((size_t)p * K + kmin) * kGallPl];
  I.Q_out_pl[toff + ((size_t)p * K + K - 1) * kGallPl] = I.Q_out_pl[toff + ((size_t)p * K + kmax) * kGallPl];
  if (tr == 0) {
    for (int k = kmin; k <= kmax; ++k)
      I.rho_out_pl[((size_t)p * K + k) * kGallPl] = rh[k] - (W(k + 1) - W(k)) * I.dt * I.rdgz[k];
    I.rho_out_pl[((size_t)p * K) * kGallPl] = I.rho_out_pl[((size_t)p * K + kmin) * kGallPl];
    I.rho_out_pl[((size_t)p * K + K - 1) * kGallPl] = I.rho_out_pl[((size_t)p * K + kmax) * kGallPl];
  }
}

// ---- halo points no list writes keep their input values (the reference never touches them)
__global__ void k_fast_carry(FastInst I) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)I.ncarry * I.K) return;
  const int p = I.carry[tid % I.ncarry], k = (int)(tid / I.ncarry);
  if (p < 0) return;
  const int l = p / I.gall, c = p % I.gall;
  const size_t off = ((size_t)l * I.K + k) * I.gall + c, tstride = (size_t)I.lall * I.K * I.gall;
  I.rho_out[off] = I.rho_in[off];
  for (int t = 0; t < I.ntr; ++t) I.Q_out[(size_t)t * tstride + off] = I.Q_in[(size_t)t * tstride + off];
}

// ---------------------------------------------------------------------------------------
template <int TX, int TY, int TG>
static cudaError_t launch_tile(const FastInst &I, cudaStream_t st) {
  const size_t smem = sizeof(TileSmem<TX, TY>);
  cudaError_t e = cudaFuncSetAttribute(k_fast_tile<TX, TY, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int ngroups = (I.ntr + TG - 1) / TG;
  const long long blocks = (long long)I.lall * I.ntx * I.nty * ngroups;
  k_fast_tile<TX, TY, TG><<<(unsigned)blocks, TX * TY, smem, st>>>(I);
  return cudaGetLastError();
}

int fast_tile_shapes(int *tx, int *ty, int *tg, int nmax) {
  static const int shapes[][3] = {{16, 16, 4}, {16, 16, 2}, {16, 8, 4}, {32, 8, 4}, {16, 16, 8}, {8, 8, 4}};
  const int n = sizeof(shapes) / sizeof(shapes[0]);
  if (tx)
    for (int i = 0; i < n; ++i) tx[i] = shapes[i][0], ty[i] = shapes[i][1], tg[i] = shapes[i][2];
  (void)nmax;
  return n;
}

cudaError_t fast_step(const FastInst &I, int shape, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                      long long &launches) {
  const long long nbt = (long long)I.nb * (I.K - 2) * I.ntr;
  k_fast_boundary<<<(unsigned)((nbt + 127) / 128), 128, 0, st>>>(I);
  if (I.K <= 48) k_fast_pole<48><<<1, 64, 0, st>>>(I);
  else if (I.K <= 128) k_fast_pole<128><<<1, 64, 0, st>>>(I);
  else return cudaErrorInvalidValue;
  if (ev0) cudaEventRecord(ev0, st);
  cudaError_t e;
  switch (shape) {
    case 0: e = launch_tile<16, 16, 4>(I, st); break;
    case 1: e = launch_tile<16, 16, 2>(I, st); break;
    case 2: e = launch_tile<16, 8, 4>(I, st); break;
    case 3: e = launch_tile<32, 8, 4>(I, st); break;
    case 4: e = launch_tile<16, 16, 8>(I, st); break;
    case 5: e = launch_tile<8, 8, 4>(I, st); break;
    default: return cudaErrorInvalidValue;
  }
  if (ev1) cudaEventRecord(ev1, st);
  const long long nc = (long long)I.ncarry * I.K;
  k_fast_carry<<<(unsigned)((nc + 127) / 128), 128, 0, st>>>(I);
  launches += 4;
  return e;
}

}  // namespace icoadv
