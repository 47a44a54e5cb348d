// C ABI of the library: context, metrics registration and the drop-in entry
// points that keep the reference subroutines' argument lists.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "capi_internal.h"

namespace icoadv {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  cudaGetLastError();  // a launch-configuration error is not sticky: do not hand it to the next call
  return ICA_ERR_CUDA;
}

void *Ctx::buf(const char *name, size_t bytes) {
  DevBuf &b = bufs[name];
  if (b.bytes < bytes) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    if (cudaMalloc(&b.ptr, bytes ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    b.bytes = bytes;
  }
  return b.ptr;
}

void Ctx::release(const char *name) {
  auto it = bufs.find(name);
  if (it == bufs.end()) return;
  if (it->second.ptr) cudaFree(it->second.ptr);
  bufs.erase(it);
}

int Ctx::need_grid(const char *what) const {
  if (topo) return ICA_OK;
  set_error(std::string(what) + ": this context was made by ica_init_regions and holds no region topology "
            "(the halo fill and the composed steps need a whole grid, ica_init)");
  return ICA_ERR_STATE;
}

int Ctx::check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  return ICA_OK;
}

}  // namespace icoadv

using namespace icoadv;

struct ica_ctx : public Ctx {};

extern "C" {

const char *ica_last_error(void) { return icoadv::g_last_error.c_str(); }

int ica_device_check(int device) {
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
  if (prop.major != 10 || prop.minor != 0) {
    set_error("device is not sm_100 (this library is built for sm_100a only)");
    return ICA_ERR_STATE;
  }
  return ICA_OK;
}

int ica_init(const ica_dims *dims, ica_ctx **out) {
  if (!dims || !out) return set_error("ica_init: NULL argument"), ICA_ERR_ARG;
  *out = nullptr;
  if (dims->glevel < 1 || dims->glevel > 11 || dims->rlevel < 0 || dims->rlevel > dims->glevel ||
      dims->vlayer < 1 || dims->vlayer > 4094)
    return set_error("ica_init: glevel/rlevel/vlayer out of range"), ICA_ERR_ARG;
  cudaError_t e = cudaSetDevice(dims->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  int rc = ica_device_check(dims->device);
  if (rc) return rc;
  ica_ctx *c = new ica_ctx();
  c->topo.reset(new Topology(dims->glevel, dims->rlevel));
  const Topology &t = *c->topo;
  c->device = dims->device;
  ica_sizes &s = c->sz;
  s.gall_1d = t.gall_1d;
  s.gall = t.gall;
  s.gmin = t.gmin;
  s.gmax = t.gmax;
  if (dims->vlayer == 1) s.kall = s.kmin = s.kmax = 1;
  else s.kall = dims->vlayer + 2, s.kmin = 2, s.kmax = dims->vlayer + 1;
  s.lall = t.nrgn;
  s.gall_pl = kGallPl;
  s.lall_pl = kLallPl;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaStreamCreate"); }
  for (int pf = 0; pf < 2; ++pf) {
    std::vector<int> d, sr;
    rc = t.build_plan(pf != 0, d, sr);
    if (rc) { delete c; return set_error("halo plan: a source is also a destination"), rc; }
    Plan &p = c->plan[pf];
    p.n = (int)d.size();
    if (cudaMalloc(&p.dst, sizeof(int) * (p.n + 1)) != cudaSuccess ||
        cudaMalloc(&p.src, sizeof(int) * (p.n + 1)) != cudaSuccess) {
      delete c;
      return set_error("cudaMalloc(plan)"), ICA_ERR_NOMEM;
    }
    cudaMemcpy(p.dst, d.data(), sizeof(int) * p.n, cudaMemcpyHostToDevice);
    cudaMemcpy(p.src, sr.data(), sizeof(int) * p.n, cudaMemcpyHostToDevice);
  }
  if (cudaMalloc(&c->d_have_sgp, sizeof(int) * t.nrgn) != cudaSuccess) {
    delete c;
    return set_error("cudaMalloc(have_sgp)"), ICA_ERR_NOMEM;
  }
  cudaMemcpy(c->d_have_sgp, t.have_sgp.data(), sizeof(int) * t.nrgn, cudaMemcpyHostToDevice);
  c->D.gall_1d = s.gall_1d;
  c->D.gall = s.gall;
  c->D.gmin = s.gmin;
  c->D.gmax = s.gmax;
  c->D.kall = s.kall;
  c->D.kmin = s.kmin;
  c->D.kmax = s.kmax;
  c->D.lall = s.lall;
  c->D.have_sgp = c->d_have_sgp;
  c->D.have_pl = 1;
  // the noalloc limiter's fixed scratch: loaded now, while the context is created, so that
  // its first call takes no device memory (with lazy module loading the array would
  // otherwise be set up inside that call)
  if (noalloc_scratch_address(&c->noalloc_scratch) != ICA_OK) c->noalloc_scratch = nullptr;
  e = cudaGetLastError();
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "ica_init"); }
  *out = c;
  return ICA_OK;
}

int ica_init_regions(int gall_1d, int kall, int kmin, int kmax, int lall, int have_pl, const int *have_sgp,
                     int device, ica_ctx **out) {
  if (!out || !have_sgp) return set_error("ica_init_regions: NULL argument"), ICA_ERR_ARG;
  *out = nullptr;
  if (gall_1d < 3 || gall_1d > 4098 || kall < 1 || kall > 4096 || kmin < 1 || kmax < kmin || kmax > kall ||
      lall < 1 || lall > 40960 || (long long)gall_1d * gall_1d * kall * lall >= (1LL << 31))
    return set_error("ica_init_regions: sizes out of range"), ICA_ERR_ARG;
  for (int l = 0; l < lall; ++l)
    if (have_sgp[l] != 0 && have_sgp[l] != 1) return set_error("ica_init_regions: have_sgp must be 0 or 1"), ICA_ERR_ARG;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  int rc = ica_device_check(device);
  if (rc) return rc;
  ica_ctx *c = new ica_ctx();
  c->device = device;
  ica_sizes &s = c->sz;
  s.gall_1d = gall_1d;
  s.gall = gall_1d * gall_1d;
  s.gmin = 2;
  s.gmax = gall_1d - 1;
  s.kall = kall, s.kmin = kmin, s.kmax = kmax;
  s.lall = lall;
  s.gall_pl = kGallPl;
  s.lall_pl = kLallPl;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaStreamCreate"); }
  if (cudaMalloc(&c->d_have_sgp, sizeof(int) * lall) != cudaSuccess) {
    delete c;
    return set_error("cudaMalloc(have_sgp)"), ICA_ERR_NOMEM;
  }
  e = cudaMemcpy(c->d_have_sgp, have_sgp, sizeof(int) * lall, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaMemcpy(have_sgp)"); }
  c->D.gall_1d = s.gall_1d, c->D.gall = s.gall, c->D.gmin = s.gmin, c->D.gmax = s.gmax;
  c->D.kall = s.kall, c->D.kmin = s.kmin, c->D.kmax = s.kmax;
  c->D.lall = s.lall;
  c->D.have_sgp = c->d_have_sgp;
  c->D.have_pl = have_pl ? 1 : 0;
  if (noalloc_scratch_address(&c->noalloc_scratch) != ICA_OK) c->noalloc_scratch = nullptr;
  e = cudaGetLastError();
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "ica_init_regions"); }
  *out = c;
  return ICA_OK;
}

int ica_finalize(ica_ctx *c) {
  if (!c) return ICA_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete c;
  return ICA_OK;
}

int ica_get_sizes(const ica_ctx *c, ica_sizes *out) {
  if (!c || !out) return ICA_ERR_ARG;
  *out = c->sz;
  return ICA_OK;
}

void *ica_stream(ica_ctx *c) { return c ? (void *)c->stream : nullptr; }
long long ica_launch_count(const ica_ctx *c) { return c ? c->launches : -1; }

int ica_set_geometry(ica_ctx *c, const double *GRD_xr, const double *GRD_xr_pl, const double *GMTR_p,
                     const double *GMTR_p_pl, const double *GMTR_t, const double *GMTR_t_pl, const double *GMTR_a,
                     const double *GMTR_a_pl) {
  if (!c || !GRD_xr || !GRD_xr_pl || !GMTR_p || !GMTR_p_pl || !GMTR_t || !GMTR_t_pl || !GMTR_a || !GMTR_a_pl)
    return set_error("ica_set_geometry: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t gl = (size_t)c->sz.gall * c->sz.lall, pl = (size_t)kGallPl * kLallPl;
  const double *h[8] = {GRD_xr, GRD_xr_pl, GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl};
  const size_t n[8] = {gl * 9, pl * 3, gl * 8, pl * 8, gl * 10, pl * 5, gl * 36, pl * 18};
  c->fast.off_ready = false;
  c->fast.off64_ready = false;
  return c->upload_geometry(h, n);
}

}  // extern "C"

namespace icoadv {

Ctx::~Ctx() {
  for (auto &kv : bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  for (auto &p : plan) {
    if (p.dst) cudaFree(p.dst);
    if (p.src) cudaFree(p.src);
  }
  for (int i = 0; i < 8; ++i) {
    if (geo64[i]) cudaFree(geo64[i]);
    if (geo32[i]) cudaFree(geo32[i]);
  }
  if (d_have_sgp) cudaFree(d_have_sgp);
  for (void *p : stepgeo)
    if (p) cudaFree(p);
  for (void *p : {(void *)fast.bsrc, (void *)fast.blist, (void *)fast.ring, (void *)fast.carry, (void *)fast.cg32,
                  (void *)fast.off32, (void *)fast.off64, (void *)fast.seam_list,
                  (void *)fast.seam_id})
    if (p) cudaFree(p);
  for (auto &ev : fast.events) cudaEventDestroy(ev.first), cudaEventDestroy(ev.second);
  if (fast.local.dst) cudaFree(fast.local.dst);
  if (fast.local.src) cudaFree(fast.local.src);
  if (stream) cudaStreamDestroy(stream);
  if (copy_in) cudaStreamDestroy(copy_in);
  if (copy_out) cudaStreamDestroy(copy_out);
}

int Ctx::copy_streams() {
  for (cudaStream_t *s : {&copy_in, &copy_out})
    if (!*s) {
      cudaError_t e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate(copy)");
    }
  return ICA_OK;
}

int Ctx::upload_geometry(const double *const h[8], const size_t n[8]) {
  std::vector<float> tmp;
  for (int i = 0; i < 8; ++i) {
    if (!geo64[i] && cudaMalloc(&geo64[i], n[i] * sizeof(double)) != cudaSuccess)
      return set_error("cudaMalloc(geometry)"), ICA_ERR_NOMEM;
    if (!geo32[i] && cudaMalloc(&geo32[i], n[i] * sizeof(float)) != cudaSuccess)
      return set_error("cudaMalloc(geometry)"), ICA_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(geo64[i], h[i], n[i] * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(geometry)");
    tmp.resize(n[i]);
    for (size_t j = 0; j < n[i]; ++j) tmp[j] = (float)h[i][j];
    e = cudaMemcpy(geo32[i], tmp.data(), n[i] * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(geometry)");
  }
  geo_n.assign(n, n + 8);
  geo_set = true;
  return ICA_OK;
}

template <> Geo<double> Ctx::geo<double>() const {
  const double *const *p = (const double *const *)geo64;
  return Geo<double>{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7]};
}
template <> Geo<float> Ctx::geo<float>() const {
  const float *const *p = (const float *const *)geo32;
  return Geo<float>{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7]};
}

// ---- device-pointer implementations (asynchronous on the context stream)
template <typename T>
int flux_dev(Ctx *c, T *flx_h, T *flx_h_pl, T *GRD_xc, T *GRD_xc_pl, const T *rho, const T *rho_pl, const T *vx,
             const T *vx_pl, const T *vy, const T *vy_pl, const T *vz, const T *vz_pl, T dt) {
  if (!c->geo_set) return set_error("horizontal_flux: geometry not registered"), ICA_ERR_STATE;
  if (!flx_h || !flx_h_pl || !GRD_xc || !GRD_xc_pl || !rho || !rho_pl || !vx || !vx_pl || !vy || !vy_pl || !vz ||
      !vz_pl)
    return set_error("horizontal_flux: NULL argument"), ICA_ERR_ARG;
  FluxIn<T> in{rho, rho_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl};
  FluxOut<T> out{flx_h, flx_h_pl, GRD_xc, GRD_xc_pl};
  launch_horizontal_flux<T>(c->D, in, out, c->geo<T>(), dt, c->stream);
  c->launches += c->D.have_pl ? 2 : 1;
  return c->check_launch("horizontal_flux");
}

template <typename T>
int comm_dev(Ctx *c, T *var, T *var_pl, int kmax, int vmax, bool pole_fill) {
  if (!var || !var_pl || kmax < 1 || vmax < 1) return set_error("COMM: bad argument"), ICA_ERR_ARG;
  int rc = c->need_grid(pole_fill ? "COMM_var" : "COMM_data_transfer");
  if (rc) return rc;
  const Plan &p = c->plan[pole_fill ? 1 : 0];
  launch_gather<T>(c->D, p.n, p.dst, p.src, kmax, vmax, var, var_pl, c->stream);
  c->launches += 1;
  return c->check_launch("COMM_data_transfer");
}

template <typename T>
int hlim_dev(Ctx *c, T *q_a, T *q_a_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ch,
             const T *ch_pl, const T *cmask, const T *cmask_pl, T *Qout_prev, T *Qout_prev_pl, const T *Qout_post,
             const T *Qout_post_pl, T *scratch_Qout, T *scratch_Qout_pl, T *scratch_Qin_pl) {
  if (!q_a || !q_a_pl || !q || !q_pl || !d || !d_pl || !ch || !ch_pl || !cmask || !cmask_pl || !Qout_prev ||
      !Qout_prev_pl || ((Qout_post == nullptr) != (Qout_post_pl == nullptr)))
    return set_error("horizontal_limiter_thuburn: bad argument"), ICA_ERR_ARG;
  if (!Qout_post) {  // the on-GPU Qout halo fill needs the whole grid
    int rc = c->need_grid("horizontal_limiter_thuburn with Qout_post = NULL");
    if (rc) return rc;
  }
  const size_t n2 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall * 2, n2p = (size_t)kGallPl * c->sz.kall * kLallPl * 2;
  LimIn<T> in{q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl};
  launch_hlim_qout<T>(c->D, in, Qout_prev, Qout_prev_pl, scratch_Qin_pl, c->stream);
  c->launches += c->D.have_pl ? 2 : 1;
  const T *Qo = Qout_post, *Qo_pl = Qout_post_pl;
  if (!Qout_post) {  // NICAM: COMM_data_transfer(Qout, Qout_pl) on a copy of the pre-fill Qout
    cudaError_t e = cudaMemcpyAsync(scratch_Qout, Qout_prev, n2 * sizeof(T), cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "horizontal_limiter_thuburn: copy of Qout");
    e = cudaMemcpyAsync(scratch_Qout_pl, Qout_prev_pl, n2p * sizeof(T), cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "horizontal_limiter_thuburn: copy of Qout_pl");
    const Plan &p = c->plan[0];
    launch_gather<T>(c->D, p.n, p.dst, p.src, c->sz.kall, 2, scratch_Qout, scratch_Qout_pl, c->stream);
    c->launches += 1;
    Qo = scratch_Qout;
    Qo_pl = scratch_Qout_pl;
  }
  launch_hlim_apply<T>(c->D, in, q_a, q_a_pl, Qo, Qo_pl, scratch_Qin_pl, c->stream);
  c->launches += c->D.have_pl ? 2 : 1;
  return c->check_launch("horizontal_limiter_thuburn");
}

template int hlim_dev<double>(Ctx *, double *, double *, const double *, const double *, const double *,
                              const double *, const double *, const double *, const double *, const double *,
                              double *, double *, const double *, const double *, double *, double *, double *);

template <typename T>
int hlim_dev_alloc(Ctx *c, T *q_a, T *q_a_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ch,
                   const T *ch_pl, const T *cmask, const T *cmask_pl, T *Qout_prev, T *Qout_prev_pl,
                   const T *Qout_post, const T *Qout_post_pl) {
  const size_t n2 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall * 2, n2p = (size_t)kGallPl * c->sz.kall * kLallPl * 2;
  T *sq = (T *)c->buf(sizeof(T) == 8 ? "lim_qout64" : "lim_qout32", n2 * sizeof(T));
  T *sqp = (T *)c->buf(sizeof(T) == 8 ? "lim_qoutpl64" : "lim_qoutpl32", n2p * sizeof(T));
  T *sqin = (T *)c->buf(sizeof(T) == 8 ? "lim_qinpl64" : "lim_qinpl32", n2p * 2 * sizeof(T));
  if (!sq || !sqp || !sqin) return set_error("horizontal_limiter_thuburn: cudaMalloc(scratch)"), ICA_ERR_NOMEM;
  return hlim_dev<T>(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl, Qout_prev, Qout_prev_pl,
                     Qout_post, Qout_post_pl, sq, sqp, sqin);
}

template <typename T>
int vlim_dev(Ctx *c, T *q_h, T *q_h_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ck,
             const T *ck_pl) {
  if (!q_h || !q_h_pl || !q || !q_pl || !d || !d_pl || !ck || !ck_pl)
    return set_error("vertical_limiter_thuburn: NULL argument"), ICA_ERR_ARG;
  launch_vlim<T>(c->D, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl, c->stream);
  if (c->D.kmax > c->D.kmin) c->launches += c->D.have_pl ? 2 : 1;
  return c->check_launch("vertical_limiter_thuburn");
}

// ---- host-pointer staging
template <typename T> struct Stage {
  Ctx *c;
  int rc = ICA_OK;
  explicit Stage(Ctx *cc) : c(cc) {}
  T *in(const char *name, const T *h, size_t n) {
    if (rc) return nullptr;
    T *d = (T *)c->buf(name, n * sizeof(T));
    if (!d) { rc = ICA_ERR_NOMEM; set_error(std::string("cudaMalloc ") + name); return nullptr; }
    if (h) {
      cudaError_t e = cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, c->stream);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(H2D)");
    }
    return d;
  }
  void out(T *h, const T *d, size_t n) {
    if (rc || !h) return;
    cudaError_t e = cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(D2H)");
  }
  int sync() {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamSynchronize");
    return rc;
  }
};

template <typename T>
int flux_host(Ctx *c, T *flx_h, T *flx_h_pl, T *GRD_xc, T *GRD_xc_pl, const T *rho, const T *rho_pl, const T *vx,
              const T *vx_pl, const T *vy, const T *vy_pl, const T *vz, const T *vz_pl, T dt) {
  if (!flx_h || !flx_h_pl || !GRD_xc || !GRD_xc_pl || !rho || !rho_pl || !vx || !vx_pl || !vy || !vy_pl || !vz ||
      !vz_pl)
    return set_error("horizontal_flux: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  Stage<T> s(c);
  T *d_rho = s.in("a0", rho, n3), *d_rho_pl = s.in("a1", rho_pl, n3p);
  T *d_vx = s.in("a2", vx, n3), *d_vx_pl = s.in("a3", vx_pl, n3p);
  T *d_vy = s.in("a4", vy, n3), *d_vy_pl = s.in("a5", vy_pl, n3p);
  T *d_vz = s.in("a6", vz, n3), *d_vz_pl = s.in("a7", vz_pl, n3p);
  T *d_f = s.in("o0", nullptr, n3 * 6), *d_fp = s.in("o1", flx_h_pl, n3p);
  T *d_x = s.in("o2", nullptr, n3 * 9), *d_xp = s.in("o3", GRD_xc_pl, n3p * 3);
  if (s.rc) return s.rc;
  int rc = flux_dev<T>(c, d_f, d_fp, d_x, d_xp, d_rho, d_rho_pl, d_vx, d_vx_pl, d_vy, d_vy_pl, d_vz, d_vz_pl, dt);
  if (rc) return rc;
  s.out(flx_h, d_f, n3 * 6);
  s.out(flx_h_pl, d_fp, n3p);
  s.out(GRD_xc, d_x, n3 * 9);
  s.out(GRD_xc_pl, d_xp, n3p * 3);
  return s.sync();
}

template <typename T>
int hlim_host(Ctx *c, T *q_a, T *q_a_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ch,
              const T *ch_pl, const T *cmask, const T *cmask_pl, T *Qout_prev, T *Qout_prev_pl, const T *Qout_post,
              const T *Qout_post_pl) {
  if (!q_a || !q_a_pl || !q || !q_pl || !d || !d_pl || !ch || !ch_pl || !cmask || !cmask_pl || !Qout_prev ||
      !Qout_prev_pl || ((Qout_post == nullptr) != (Qout_post_pl == nullptr)))
    return set_error("horizontal_limiter_thuburn: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  Stage<T> s(c);
  T *d_qa = s.in("a0", q_a, n3 * 6), *d_qap = s.in("a1", q_a_pl, n3p);
  T *d_q = s.in("a2", q, n3), *d_qp = s.in("a3", q_pl, n3p);
  T *d_d = s.in("a4", d, n3), *d_dp = s.in("a5", d_pl, n3p);
  T *d_ch = s.in("a6", ch, n3 * 6), *d_chp = s.in("a7", ch_pl, n3p);
  T *d_cm = s.in("a8", cmask, n3 * 6), *d_cmp = s.in("a9", cmask_pl, n3p);
  T *d_qo = s.in("o0", nullptr, n3 * 2), *d_qop = s.in("o1", nullptr, n3p * 2);
  T *d_po = Qout_post ? s.in("a10", Qout_post, n3 * 2) : nullptr;
  T *d_pop = Qout_post ? s.in("a11", Qout_post_pl, n3p * 2) : nullptr;
  if (s.rc) return s.rc;
  int rc = hlim_dev_alloc<T>(c, d_qa, d_qap, d_q, d_qp, d_d, d_dp, d_ch, d_chp, d_cm, d_cmp, d_qo, d_qop, d_po,
                             d_pop);
  if (rc) return rc;
  s.out(q_a, d_qa, n3 * 6);
  s.out(q_a_pl, d_qap, n3p);
  s.out(Qout_prev, d_qo, n3 * 2);
  s.out(Qout_prev_pl, d_qop, n3p * 2);
  return s.sync();
}

template <typename T>
int vlim_host(Ctx *c, T *q_h, T *q_h_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ck,
              const T *ck_pl) {
  if (!q_h || !q_h_pl || !q || !q_pl || !d || !d_pl || !ck || !ck_pl)
    return set_error("vertical_limiter_thuburn: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  Stage<T> s(c);
  T *d_qh = s.in("a0", q_h, n3), *d_qhp = s.in("a1", q_h_pl, n3p);
  T *d_q = s.in("a2", q, n3), *d_qp = s.in("a3", q_pl, n3p);
  T *d_d = s.in("a4", d, n3), *d_dp = s.in("a5", d_pl, n3p);
  T *d_ck = s.in("a6", ck, n3 * 2), *d_ckp = s.in("a7", ck_pl, n3p * 2);
  if (s.rc) return s.rc;
  int rc = vlim_dev<T>(c, d_qh, d_qhp, d_q, d_qp, d_d, d_dp, d_ck, d_ckp);
  if (rc) return rc;
  s.out(q_h, d_qh, n3);
  s.out(q_h_pl, d_qhp, n3p);
  return s.sync();
}

template <typename T>
int comm_host(Ctx *c, T *var, T *var_pl, int kmax, int vmax, bool pole_fill) {
  if (!var || !var_pl || kmax < 1 || vmax < 1) return set_error("COMM: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->sz.gall * kmax * c->sz.lall * vmax, np = (size_t)kGallPl * kmax * kLallPl * vmax;
  Stage<T> s(c);
  T *dv = s.in("a0", var, n), *dp = s.in("a1", var_pl, np);
  if (s.rc) return s.rc;
  int rc = comm_dev<T>(c, dv, dp, kmax, vmax, pole_fill);
  if (rc) return rc;
  s.out(var, dv, n);
  s.out(var_pl, dp, np);
  return s.sync();
}

}  // namespace icoadv

#define CTX_OK(c) \
  if (!(c)) return set_error("NULL context"), ICA_ERR_ARG

extern "C" {

int ica_horizontal_flux(ica_ctx *c, double *a, double *b, double *x, double *y, const double *r, const double *rp,
                        const double *vx, const double *vxp, const double *vy, const double *vyp, const double *vz,
                        const double *vzp, double dt) {
  CTX_OK(c);
  return flux_host<double>(c, a, b, x, y, r, rp, vx, vxp, vy, vyp, vz, vzp, dt);
}
int ica_horizontal_flux_f32(ica_ctx *c, float *a, float *b, float *x, float *y, const float *r, const float *rp,
                            const float *vx, const float *vxp, const float *vy, const float *vyp, const float *vz,
                            const float *vzp, float dt) {
  CTX_OK(c);
  return flux_host<float>(c, a, b, x, y, r, rp, vx, vxp, vy, vyp, vz, vzp, dt);
}
int ica_horizontal_flux_dev(ica_ctx *c, double *a, double *b, double *x, double *y, const double *r,
                            const double *rp, const double *vx, const double *vxp, const double *vy,
                            const double *vyp, const double *vz, const double *vzp, double dt) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  return flux_dev<double>(c, a, b, x, y, r, rp, vx, vxp, vy, vyp, vz, vzp, dt);
}

int ica_horizontal_limiter_thuburn(ica_ctx *c, double *q_a, double *q_a_pl, const double *q, const double *q_pl,
                                   const double *d, const double *d_pl, const double *ch, const double *ch_pl,
                                   const double *cm, const double *cm_pl, double *qo, double *qo_pl,
                                   const double *qp, const double *qp_pl) {
  CTX_OK(c);
  return hlim_host<double>(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, qp, qp_pl);
}
int ica_horizontal_limiter_thuburn_f32(ica_ctx *c, float *q_a, float *q_a_pl, const float *q, const float *q_pl,
                                       const float *d, const float *d_pl, const float *ch, const float *ch_pl,
                                       const float *cm, const float *cm_pl, float *qo, float *qo_pl,
                                       const float *qp, const float *qp_pl) {
  CTX_OK(c);
  return hlim_host<float>(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, qp, qp_pl);
}
int ica_horizontal_limiter_thuburn_dev(ica_ctx *c, double *q_a, double *q_a_pl, const double *q,
                                       const double *q_pl, const double *d, const double *d_pl, const double *ch,
                                       const double *ch_pl, const double *cm, const double *cm_pl, double *qo,
                                       double *qo_pl, const double *qp, const double *qp_pl) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  return hlim_dev_alloc<double>(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, qp, qp_pl);
}

int ica_vertical_limiter_thuburn(ica_ctx *c, double *q_h, double *q_h_pl, const double *q, const double *q_pl,
                                 const double *d, const double *d_pl, const double *ck, const double *ck_pl) {
  CTX_OK(c);
  return vlim_host<double>(c, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl);
}
int ica_vertical_limiter_thuburn_f32(ica_ctx *c, float *q_h, float *q_h_pl, const float *q, const float *q_pl,
                                     const float *d, const float *d_pl, const float *ck, const float *ck_pl) {
  CTX_OK(c);
  return vlim_host<float>(c, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl);
}
int ica_vertical_limiter_thuburn_dev(ica_ctx *c, double *q_h, double *q_h_pl, const double *q, const double *q_pl,
                                     const double *d, const double *d_pl, const double *ck, const double *ck_pl) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  return vlim_dev<double>(c, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl);
}

int ica_comm_data_transfer(ica_ctx *c, double *var, double *var_pl, int kmax, int vmax) {
  CTX_OK(c);
  return comm_host<double>(c, var, var_pl, kmax, vmax, false);
}
int ica_comm_data_transfer_f32(ica_ctx *c, float *var, float *var_pl, int kmax, int vmax) {
  CTX_OK(c);
  return comm_host<float>(c, var, var_pl, kmax, vmax, false);
}
int ica_comm_data_transfer_dev(ica_ctx *c, double *var, double *var_pl, int kmax, int vmax) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  return comm_dev<double>(c, var, var_pl, kmax, vmax, false);
}
int ica_comm_var(ica_ctx *c, double *var, double *var_pl, int kmax, int vmax) {
  CTX_OK(c);
  return comm_host<double>(c, var, var_pl, kmax, vmax, true);
}
int ica_comm_var_dev(ica_ctx *c, double *var, double *var_pl, int kmax, int vmax) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  return comm_dev<double>(c, var, var_pl, kmax, vmax, true);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// composed step
namespace icoadv {

int Ctx::step_ctx(StepCtx &S) {
  int rc0 = need_grid("advect_step");
  if (rc0) return rc0;
  if (!geo_set || !stepgeo_set) return set_error("advect_step: geometry not registered"), ICA_ERR_STATE;
  const size_t n3 = (size_t)sz.gall * sz.kall * sz.lall, n3p = (size_t)kGallPl * sz.kall * kLallPl;
  S.D = D;
  S.geo = geo<double>();
  S.plan = DevPlan{plan[0].n, plan[0].dst, plan[0].src};
  const double *const *g = (const double *const *)stepgeo;
  S.GRD_x = g[0], S.GRD_x_pl = g[1], S.cg = g[2], S.cg_pl = g[3], S.rdgz = g[4], S.afact = g[5], S.bfact = g[6];
  struct B {
    double **p;
    const char *name;
    size_t n;
  } bl[] = {{&S.flx, "st_flx", n3 * 6}, {&S.flx_pl, "st_flxp", n3p}, {&S.xc, "st_xc", n3 * 9},
            {&S.xc_pl, "st_xcp", n3p * 3}, {&S.ch, "st_ch", n3 * 6}, {&S.ch_pl, "st_chp", n3p},
            {&S.cm, "st_cm", n3 * 6}, {&S.cm_pl, "st_cmp", n3p}, {&S.zero, "st_zero", n3},
            {&S.zero_pl, "st_zerop", n3p}, {&S.q, "st_q", n3}, {&S.q_pl, "st_qp", n3p},
            {&S.grad, "st_grad", n3 * 3}, {&S.grad_pl, "st_gradp", n3p * 3}, {&S.qa, "st_qa", n3 * 6},
            {&S.qa_pl, "st_qap", n3p}, {&S.qout, "st_qout", n3 * 2}, {&S.qout_pl, "st_qoutp", n3p * 2},
            {&S.qin_pl, "st_qinp", n3p * 4}};
  bool fresh_zero = bufs.find("st_zero") == bufs.end();
  for (auto &b : bl) {
    *b.p = (double *)buf(b.name, b.n * sizeof(double));
    if (!*b.p) return set_error(std::string("cudaMalloc ") + b.name), ICA_ERR_NOMEM;
  }
  if (fresh_zero) {
    cudaMemsetAsync(S.zero, 0, n3 * sizeof(double), stream);
    cudaMemsetAsync(S.zero_pl, 0, n3p * sizeof(double), stream);
  }
  return ICA_OK;
}

}  // namespace icoadv

extern "C" {

int ica_set_step_geometry(ica_ctx *c, const double *GRD_x, const double *GRD_x_pl, const double *coef_grad,
                          const double *coef_grad_pl, const double *rdgz, const double *afact, const double *bfact) {
  CTX_OK(c);
  if (!GRD_x || !GRD_x_pl || !coef_grad || !coef_grad_pl || !rdgz || !afact || !bfact)
    return set_error("ica_set_step_geometry: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t gl = (size_t)c->sz.gall * c->sz.lall;
  const double *h[7] = {GRD_x, GRD_x_pl, coef_grad, coef_grad_pl, rdgz, afact, bfact};
  const size_t n[7] = {gl * 3, (size_t)kGallPl * kLallPl * 3, gl * 21, (size_t)6 * 3 * kLallPl,
                       (size_t)c->sz.kall, (size_t)c->sz.kall, (size_t)c->sz.kall};
  for (int i = 0; i < 7; ++i) {
    if (!c->stepgeo[i] && cudaMalloc(&c->stepgeo[i], n[i] * sizeof(double)) != cudaSuccess)
      return set_error("cudaMalloc(step geometry)"), ICA_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(c->stepgeo[i], h[i], n[i] * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(step geometry)");
  }
  // FP32 copy of the gradient coefficients for the batched path
  std::vector<float> cg32(n[2]);
  for (size_t j = 0; j < n[2]; ++j) cg32[j] = (float)coef_grad[j];
  if (!c->fast.cg32 && cudaMalloc(&c->fast.cg32, n[2] * sizeof(float)) != cudaSuccess)
    return set_error("cudaMalloc(coef_grad fp32)"), ICA_ERR_NOMEM;
  cudaError_t e = cudaMemcpy(c->fast.cg32, cg32.data(), n[2] * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(coef_grad fp32)");
  c->stepgeo_set = true;
  c->fast.off_ready = false;
  c->fast.off64_ready = false;
  return ICA_OK;
}

int ica_advect_step_dev(ica_ctx *c, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq,
                        double *rhogq_pl, const double *vx, const double *vx_pl, const double *vy,
                        const double *vy_pl, const double *vz, const double *vz_pl, const double *w,
                        const double *w_pl) {
  CTX_OK(c);
  if (ntr < 1 || !rhog || !rhog_pl || !rhogq || !rhogq_pl || !vx || !vx_pl || !vy || !vy_pl || !vz || !vz_pl || !w ||
      !w_pl)
    return set_error("ica_advect_step: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  StepCtx S;
  int rc = c->step_ctx(S);
  if (rc) return rc;
  rc = step_plain(S, ntr, dt, rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl, c->stream,
                  c->launches);
  if (rc) return set_error("ica_advect_step: kall above 128"), rc;
  return c->check_launch("ica_advect_step");
}

int ica_advect_step(ica_ctx *c, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                    const double *vx, const double *vx_pl, const double *vy, const double *vy_pl, const double *vz,
                    const double *vz_pl, const double *w, const double *w_pl) {
  CTX_OK(c);
  if (ntr < 1 || !rhog || !rhog_pl || !rhogq || !rhogq_pl || !vx || !vx_pl || !vy || !vy_pl || !vz || !vz_pl || !w ||
      !w_pl)
    return set_error("ica_advect_step: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  Stage<double> s(c);
  double *d_r = s.in("h0", rhog, n3), *d_rp = s.in("h1", rhog_pl, n3p);
  double *d_q = s.in("h2", rhogq, n3 * ntr), *d_qp = s.in("h3", rhogq_pl, n3p * ntr);
  double *d_x = s.in("h4", vx, n3), *d_xp = s.in("h5", vx_pl, n3p);
  double *d_y = s.in("h6", vy, n3), *d_yp = s.in("h7", vy_pl, n3p);
  double *d_z = s.in("h8", vz, n3), *d_zp = s.in("h9", vz_pl, n3p);
  double *d_w = s.in("h10", w, n3), *d_wp = s.in("h11", w_pl, n3p);
  if (s.rc) return s.rc;
  int rc = ica_advect_step_dev(c, ntr, dt, d_r, d_rp, d_q, d_qp, d_x, d_xp, d_y, d_yp, d_z, d_zp, d_w, d_wp);
  if (rc) return rc;
  s.out(rhog, d_r, n3);
  s.out(rhog_pl, d_rp, n3p);
  s.out(rhogq, d_q, n3 * ntr);
  s.out(rhogq_pl, d_qp, n3p * ntr);
  return s.sync();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// adjoint of the composed step, and multi-step runs with step checkpointing
#include "adjoint.cuh"

namespace icoadv {

static int adj_scratch(Ctx *c, AdjScratch &A) {
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  struct B {
    double **p;
    const char *name;
    size_t n;
  } bl[] = {{&A.rh, "adj_rh", n3},         {&A.rh_pl, "adj_rhp", n3p},     {&A.qa1, "adj_tr", 8 * n3},
            {&A.qa1_pl, "adj_qa1p", n3p},  {&A.Qh_pl, "adj_Qhp", n3p},     {&A.a_q_pl, "adj_aqp", n3p},
            {&A.a_flx, "adj_aflx", 6 * n3}, {&A.a_flx_pl, "adj_aflxp", n3p}, {&A.a_xc, "adj_axc", 9 * n3},
            {&A.a_xc_pl, "adj_axcp", 3 * n3p}, {&A.a_ch, "adj_ach", 6 * n3}, {&A.a_ch_pl, "adj_achp", n3p},
            {&A.a_rh, "adj_arh", n3},      {&A.a_rh_pl, "adj_arhp", n3p},  {&A.a_gr, "adj_agr", 3 * n3},
            {&A.a_gr_pl, "adj_agrp", 3 * n3p}, {&A.a_qo, "adj_aqo", 2 * n3}, {&A.a_qo_pl, "adj_aqop", 2 * n3p}};
  for (auto &b : bl) {
    *b.p = (double *)c->buf(b.name, b.n * sizeof(double));
    if (!*b.p) return set_error(std::string("cudaMalloc ") + b.name), ICA_ERR_NOMEM;
  }
  // qa1 | Qh | a_q are one block, reused as the 8 triangle-adjoint fields after the tracers
  A.Qh = A.qa1 + 6 * n3;
  A.a_q = A.qa1 + 7 * n3;
  A.aT = A.qa1;
  return ICA_OK;
}

// one state = rhog | rhog_pl | rhogq | rhogq_pl
struct StateView {
  double *r, *rp, *q, *qp;
};
static size_t state_doubles(const Ctx *c, int ntr) {
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  return (size_t)(ntr + 1) * (n3 + n3p);
}
static StateView state_at(const Ctx *c, double *base, int ntr) {
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  return StateView{base, base + n3, base + n3 + n3p, base + n3 + n3p + ntr * n3};
}
static void copy_state(const Ctx *c, const StateView &d, const double *r, const double *rp, const double *q,
                       const double *qp, int ntr) {
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  const size_t B = sizeof(double);
  cudaMemcpyAsync(d.r, r, n3 * B, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(d.rp, rp, n3p * B, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(d.q, q, ntr * n3 * B, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(d.qp, qp, ntr * n3p * B, cudaMemcpyDeviceToDevice, c->stream);
}

}  // namespace icoadv

extern "C" {

int ica_advect_step_adjoint_dev(ica_ctx *c, int ntr, double dt, const double *rhog, const double *rhog_pl,
                                const double *rhogq, const double *rhogq_pl, const double *vx, const double *vx_pl,
                                const double *vy, const double *vy_pl, const double *vz, const double *vz_pl,
                                const double *w, const double *w_pl, double *a_rhog, double *a_rhog_pl,
                                double *a_rhogq, double *a_rhogq_pl, double *a_vx, double *a_vx_pl, double *a_vy,
                                double *a_vy_pl, double *a_vz, double *a_vz_pl) {
  CTX_OK(c);
  const void *ptrs[] = {rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl,
                        a_rhog, a_rhog_pl, a_rhogq, a_rhogq_pl, a_vx, a_vx_pl, a_vy, a_vy_pl, a_vz, a_vz_pl};
  for (const void *p : ptrs)
    if (!p) return set_error("ica_advect_step_adjoint: NULL argument"), ICA_ERR_ARG;
  if (ntr < 1) return set_error("ica_advect_step_adjoint: ntr < 1"), ICA_ERR_ARG;
  if (c->sz.kall < 4 || c->sz.kall > 128) return set_error("ica_advect_step_adjoint: needs 4 <= kall <= 128"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  StepCtx S;
  AdjScratch A;
  int rc = c->step_ctx(S);
  if (!rc) rc = adj_scratch(c, A);
  if (rc) return rc;
  rc = step_adjoint(S, A, ntr, dt, rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl, a_rhog,
                    a_rhog_pl, a_rhogq, a_rhogq_pl, a_vx, a_vx_pl, a_vy, a_vy_pl, a_vz, a_vz_pl, c->stream,
                    c->launches);
  if (rc) return set_error("ica_advect_step_adjoint: bad vertical grid"), rc;
  return c->check_launch("ica_advect_step_adjoint");
}

int ica_advect_step_adjoint(ica_ctx *c, int ntr, double dt, const double *rhog, const double *rhog_pl,
                            const double *rhogq, const double *rhogq_pl, const double *vx, const double *vx_pl,
                            const double *vy, const double *vy_pl, const double *vz, const double *vz_pl,
                            const double *w, const double *w_pl, double *a_rhog, double *a_rhog_pl, double *a_rhogq,
                            double *a_rhogq_pl, double *a_vx, double *a_vx_pl, double *a_vy, double *a_vy_pl,
                            double *a_vz, double *a_vz_pl) {
  CTX_OK(c);
  if (ntr < 1 || !rhog || !rhog_pl || !rhogq || !rhogq_pl || !vx || !vx_pl || !vy || !vy_pl || !vz || !vz_pl || !w ||
      !w_pl || !a_rhog || !a_rhog_pl || !a_rhogq || !a_rhogq_pl || !a_vx || !a_vx_pl || !a_vy || !a_vy_pl || !a_vz ||
      !a_vz_pl)
    return set_error("ica_advect_step_adjoint: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  Stage<double> s(c);
  const double *d[12] = {s.in("h0", rhog, n3),   s.in("h1", rhog_pl, n3p), s.in("h2", rhogq, n3 * ntr),
                         s.in("h3", rhogq_pl, n3p * ntr), s.in("h4", vx, n3), s.in("h5", vx_pl, n3p),
                         s.in("h6", vy, n3),     s.in("h7", vy_pl, n3p),   s.in("h8", vz, n3),
                         s.in("h9", vz_pl, n3p), s.in("h10", w, n3),       s.in("h11", w_pl, n3p)};
  double *a[10] = {s.in("j0", a_rhog, n3), s.in("j1", a_rhog_pl, n3p), s.in("j2", a_rhogq, n3 * ntr),
                   s.in("j3", a_rhogq_pl, n3p * ntr), s.in("j4", a_vx, n3), s.in("j5", a_vx_pl, n3p),
                   s.in("j6", a_vy, n3), s.in("j7", a_vy_pl, n3p), s.in("j8", a_vz, n3), s.in("j9", a_vz_pl, n3p)};
  if (s.rc) return s.rc;
  int rc = ica_advect_step_adjoint_dev(c, ntr, dt, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], d[10],
                                       d[11], a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9]);
  if (rc) return rc;
  double *h[10] = {a_rhog, a_rhog_pl, a_rhogq, a_rhogq_pl, a_vx, a_vx_pl, a_vy, a_vy_pl, a_vz, a_vz_pl};
  const size_t n[10] = {n3, n3p, n3 * ntr, n3p * ntr, n3, n3p, n3, n3p, n3, n3p};
  for (int i = 0; i < 10; ++i) s.out(h[i], a[i], n[i]);
  return s.sync();
}

int ica_adjoint_record(ica_ctx *c, int ntr, double dt, int nsteps, int every, double *rhog, double *rhog_pl,
                       double *rhogq, double *rhogq_pl, const double *vx, const double *vx_pl, const double *vy,
                       const double *vy_pl, const double *vz, const double *vz_pl, const double *w,
                       const double *w_pl) {
  CTX_OK(c);
  if (ntr < 1 || nsteps < 1 || every < 1 || !rhog || !rhog_pl || !rhogq || !rhogq_pl || !vx || !vx_pl || !vy ||
      !vy_pl || !vz || !vz_pl || !w || !w_pl)
    return set_error("ica_adjoint_record: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  c->tape = AdjTape{};
  StepCtx S;
  int rc = c->step_ctx(S);
  if (rc) return rc;
  const int ncp = (nsteps + every - 1) / every;
  const size_t sd = state_doubles(c, ntr);
  double *ck = (double *)c->buf("adj_ckpt", (size_t)ncp * sd * sizeof(double));
  if (!ck) return set_error("ica_adjoint_record: cudaMalloc of the checkpoints"), ICA_ERR_NOMEM;
  for (int s = 0; s < nsteps; ++s) {
    if (s % every == 0) copy_state(c, state_at(c, ck + (size_t)(s / every) * sd, ntr), rhog, rhog_pl, rhogq, rhogq_pl, ntr);
    rc = step_plain(S, ntr, dt, rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl, c->stream,
                    c->launches);
    if (rc) return set_error("ica_adjoint_record: kall above 128"), rc;
  }
  c->tape = AdjTape{true, ntr, nsteps, every, dt};
  return c->check_launch("ica_adjoint_record");
}

int ica_adjoint_sweep(ica_ctx *c, const double *vx, const double *vx_pl, const double *vy, const double *vy_pl,
                      const double *vz, const double *vz_pl, const double *w, const double *w_pl, double *a_rhog,
                      double *a_rhog_pl, double *a_rhogq, double *a_rhogq_pl, double *a_vx, double *a_vx_pl,
                      double *a_vy, double *a_vy_pl, double *a_vz, double *a_vz_pl) {
  CTX_OK(c);
  const void *ptrs[] = {vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl, a_rhog, a_rhog_pl, a_rhogq, a_rhogq_pl,
                        a_vx, a_vx_pl, a_vy, a_vy_pl, a_vz, a_vz_pl};
  for (const void *p : ptrs)
    if (!p) return set_error("ica_adjoint_sweep: NULL argument"), ICA_ERR_ARG;
  if (!c->tape.ready) return set_error("ica_adjoint_sweep: no recorded run"), ICA_ERR_STATE;
  if (c->sz.kall < 4 || c->sz.kall > 128) return set_error("ica_adjoint_sweep: needs 4 <= kall <= 128"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  const AdjTape T = c->tape;
  StepCtx S;
  AdjScratch A;
  int rc = c->step_ctx(S);
  if (!rc) rc = adj_scratch(c, A);
  if (rc) return rc;
  const size_t sd = state_doubles(c, T.ntr);
  double *ck = (double *)c->buf("adj_ckpt", 0);
  if (!ck) return set_error("ica_adjoint_sweep: no recorded run"), ICA_ERR_STATE;
  double *seg = T.every > 1 ? (double *)c->buf("adj_seg", (size_t)(T.every - 1) * sd * sizeof(double)) : nullptr;
  if (T.every > 1 && !seg) return set_error("ica_adjoint_sweep: cudaMalloc of the segment states"), ICA_ERR_NOMEM;
  const int ncp = (T.nsteps + T.every - 1) / T.every;
  std::vector<StateView> st((size_t)T.every);
  for (int g = ncp - 1; g >= 0; --g) {
    const int s0 = g * T.every, L = std::min(T.every, T.nsteps - s0);
    st[0] = state_at(c, ck + (size_t)g * sd, T.ntr);
    for (int u = 1; u < L; ++u) {  // recompute the segment from its checkpoint
      st[u] = state_at(c, seg + (size_t)(u - 1) * sd, T.ntr);
      copy_state(c, st[u], st[u - 1].r, st[u - 1].rp, st[u - 1].q, st[u - 1].qp, T.ntr);
      rc = step_plain(S, T.ntr, T.dt, st[u].r, st[u].rp, st[u].q, st[u].qp, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl,
                      c->stream, c->launches);
      if (rc) return set_error("ica_adjoint_sweep: kall above 128"), rc;
    }
    for (int u = L - 1; u >= 0; --u) {
      rc = step_adjoint(S, A, T.ntr, T.dt, st[u].r, st[u].rp, st[u].q, st[u].qp, vx, vx_pl, vy, vy_pl, vz, vz_pl, w,
                        w_pl, a_rhog, a_rhog_pl, a_rhogq, a_rhogq_pl, a_vx, a_vx_pl, a_vy, a_vy_pl, a_vz, a_vz_pl,
                        c->stream, c->launches);
      if (rc) return set_error("ica_adjoint_sweep: bad vertical grid"), rc;
    }
  }
  return c->check_launch("ica_adjoint_sweep");
}

int ica_adjoint_release(ica_ctx *c) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (const char *n : {"adj_ckpt", "adj_seg", "adj_rh", "adj_rhp", "adj_tr", "adj_qa1p", "adj_Qhp", "adj_aqp",
                        "adj_aflx", "adj_aflxp", "adj_axc", "adj_axcp", "adj_ach", "adj_achp", "adj_arh", "adj_arhp",
                        "adj_agr", "adj_agrp", "adj_aqo", "adj_aqop"})
    c->release(n);
  c->tape = AdjTape{};
  return ICA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batched path
#include "fast_kernels.cuh"

namespace icoadv {

// Boundary tables of the batched path: which cells' gradient / Qout come from the
// boundary pass (region-boundary cells, halo cells through the COMM plan, pole centres).
// Boundary-value tables of the batched step: bsrc (lall*gall) gives each region point its
// boundary index (>= 0: a region-boundary cell, or the halo point's source; -1 an interior cell
// off the region boundary; -2 a halo point no list writes), blist (nb) each boundary index's
// point (the region-boundary cells, then the two pole centres) and ring (2*5) the boundary
// index feeding each pole ring slot.
static int fast_boundary_tables(const Topology &t, std::vector<int> &bsrc, std::vector<int> &blist,
                                std::vector<int> &ring) {
  const int G = t.gall_1d, gall = t.gall, L = t.nrgn, g0 = t.gmin, g1 = t.gmax;
  const int npt = L * gall;
  bsrc.assign((size_t)L * gall, -1);
  blist.clear();
  for (int l = 0; l < L; ++l)
    for (int j = 1; j <= G; ++j)
      for (int i = 1; i <= G; ++i) {
        const int c = l * gall + (j - 1) * G + (i - 1);
        const bool in = i >= g0 && i <= g1 && j >= g0 && j <= g1;
        if (!in) bsrc[c] = -2;
        else if (i == g0 || i == g1 || j == g0 || j == g1) {
          bsrc[c] = (int)blist.size();
          blist.push_back(c);
        }
      }
  const int nbr = (int)blist.size();
  blist.push_back(npt + 0);
  blist.push_back(npt + kGallPl);
  ring.assign(2 * kVlink, -1);
  std::vector<int> d, s;
  int rc = t.build_plan(false, d, s);
  if (rc) return rc;
  for (size_t e = 0; e < d.size(); ++e) {
    int b;
    if (s[e] < npt) {
      b = bsrc[s[e]];
      if (b < 0) return set_error("fast tables: halo source is not a boundary cell"), ICA_ERR_INTERNAL;
    } else {
      const int q = s[e] - npt;
      if (q % kGallPl != 0) return set_error("fast tables: halo source is a pole ring point"), ICA_ERR_INTERNAL;
      b = nbr + q / kGallPl;
    }
    if (d[e] < npt) bsrc[d[e]] = b;
    else {
      const int q = d[e] - npt, p = q / kGallPl, v = q % kGallPl;
      if (v >= 1) ring[p * kVlink + (v - 1)] = b;
    }
  }
  for (int x : ring)
    if (x < 0) return set_error("fast tables: pole ring slot without a source"), ICA_ERR_INTERNAL;
  return ICA_OK;
}

int Ctx::build_fast_tables() {
  if (fast.built) return ICA_OK;
  const Topology &t = *topo;
  const int G = t.gall_1d, gall = t.gall, L = t.nrgn, g0 = t.gmin, g1 = t.gmax;
  const int npt = L * gall;
  std::vector<int> bsrc, blist, ring;
  int rc = fast_boundary_tables(t, bsrc, blist, ring);
  if (rc) return rc;
  // halo points no list writes (region corners at rlevel 0): the reference leaves them as they were
  std::vector<int> carry;
  for (int c = 0; c < npt; ++c)
    if (bsrc[c] == -2) carry.push_back(c);
  if (carry.empty()) carry.push_back(-1);  // keeps the device table non-empty; the kernel skips it
  // seam faces: every face of horizontal_flux's loops (mod_src_tracer.f90:235-309) with a halo cell
  std::vector<int> seam_list, seam_id((size_t)L * gall * 3, -1);
  auto inner = [&](int i, int j) { return i >= g0 && i <= g1 && j >= g0 && j <= g1; };
  for (int l = 0; l < L; ++l)
    for (int j = 1; j <= G; ++j)
      for (int i = 1; i <= G; ++i)
        for (int a = 0; a < 3; ++a) {
          const bool ex = (a == 0) ? (j >= g0 && j <= g1 && i >= g0 - 1 && i <= g1)
                        : (a == 1) ? (i >= g0 - 1 && i <= g1 && j >= g0 - 1 && j <= g1)
                                   : (i >= g0 && i <= g1 && j >= g0 - 1 && j <= g1);
          const int ni = (a < 2) ? i + 1 : i, nj = (a > 0) ? j + 1 : j;
          if (!ex || (inner(i, j) && inner(ni, nj))) continue;
          const int code = (l * gall + (j - 1) * G + (i - 1)) * 3 + a;
          seam_id[code] = (int)seam_list.size();
          seam_list.push_back(code);
        }
  fast.nb = (int)blist.size();
  fast.ncarry = (int)carry.size();
  fast.ns = (int)seam_list.size();
  if (cudaMalloc(&fast.bsrc, bsrc.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&fast.blist, blist.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&fast.ring, ring.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&fast.carry, carry.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&fast.seam_list, seam_list.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&fast.seam_id, seam_id.size() * sizeof(int)) != cudaSuccess)
    return set_error("cudaMalloc(fast tables)"), ICA_ERR_NOMEM;
  cudaMemcpy(fast.bsrc, bsrc.data(), bsrc.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(fast.blist, blist.data(), blist.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(fast.ring, ring.data(), ring.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(fast.carry, carry.data(), carry.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(fast.seam_list, seam_list.data(), seam_list.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(fast.seam_id, seam_id.data(), seam_id.size() * sizeof(int), cudaMemcpyHostToDevice);
  fast.built = true;
  return ICA_OK;
}

int Ctx::fast_inst(FastInst &I, int ntr, double dt, bool f64) {
  I = FastInst{};
  int rc0 = need_grid("advect_fast");
  if (rc0) return rc0;
  if (!geo_set || !stepgeo_set) return set_error("advect_fast: geometry not registered"), ICA_ERR_STATE;
  if (sz.kall < 4 || sz.kall > 128) return set_error("advect_fast: kall must be in [4, 128]"), ICA_ERR_ARG;
  if (3LL * sz.lall * sz.kall * sz.gall >= (1LL << 31))  // 32-bit face-level indices in the kernels
    return set_error("advect_fast: grid too large (3 * lall * kall * gall >= 2^31)"), ICA_ERR_ARG;
  int rc = build_fast_tables();
  if (rc) return rc;
  int tx[16], ty[16], tg[16];
  const int ns = fast_tile_shapes(tx, ty, tg, sz.gmax - sz.gmin + 1);
  if (fast.shape < 0 || fast.shape >= ns) fast.shape = 0;
  const int nmax = sz.gmax - sz.gmin + 1;
  I.G = sz.gall_1d, I.gall = sz.gall, I.gmin = sz.gmin, I.gmax = sz.gmax;
  I.K = sz.kall, I.kmin = sz.kmin, I.kmax = sz.kmax, I.lall = sz.lall, I.ntr = ntr;
  I.ntx = (nmax + tx[fast.shape] - 1) / tx[fast.shape];
  I.nty = (nmax + ty[fast.shape] - 1) / ty[fast.shape];
  I.dt = dt;
  I.have_sgp = d_have_sgp;
  const double *const *g = (const double *const *)geo64;
  I.GRD_xr = g[0], I.GRD_xr_pl = g[1], I.GMTR_p = g[2], I.GMTR_p_pl = g[3], I.GMTR_t = g[4], I.GMTR_t_pl = g[5];
  I.GMTR_a = g[6], I.GMTR_a_pl = g[7];
  const double *const *sg = (const double *const *)stepgeo;
  I.GRD_x = sg[0], I.GRD_x_pl = sg[1], I.cg = sg[2], I.cg_pl = sg[3], I.rdgz = sg[4], I.afact = sg[5], I.bfact = sg[6];
  I.cg32 = fast.cg32;
  if (!fast.off_ready) {
    const size_t noff = (size_t)sz.lall * (kOffPlanes + kFaceGeoPlanes) * sz.gall;
    if (!fast.off32 && cudaMalloc(&fast.off32, noff * sizeof(float)) != cudaSuccess)
      return set_error("cudaMalloc(fast remap offsets)"), ICA_ERR_NOMEM;
    cudaError_t e = fast_build_offsets(I, fast.off32, stream);
    if (e != cudaSuccess) return cuda_fail(e, "fast remap offsets");
    fast.off_ready = true;
  }
  I.off32 = fast.off32;
  I.f64 = f64 ? 1 : 0;
  if (f64 && !fast.off64_ready) {
    const size_t noff = (size_t)sz.lall * (kOffPlanes + kFaceGeoPlanes) * sz.gall;
    if (!fast.off64 && cudaMalloc(&fast.off64, noff * sizeof(double)) != cudaSuccess)
      return set_error("cudaMalloc(fast remap offsets, FP64)"), ICA_ERR_NOMEM;
    cudaError_t e = fast_build_offsets64(I, fast.off64, stream);
    if (e != cudaSuccess) return cuda_fail(e, "fast remap offsets (FP64)");
    fast.off64_ready = true;
  }
  I.off64 = fast.off64;
  I.bsrc = fast.bsrc, I.blist = fast.blist, I.pole_ring_b = fast.ring, I.nb = fast.nb;
  I.carry = fast.carry, I.ncarry = fast.ncarry;
  const size_t nbb = (size_t)ntr * sz.kall * fast.nb * 5;
  I.bbuf = (double *)buf("fast_bbuf", nbb * sizeof(double));
  if (!I.bbuf) return set_error("cudaMalloc(fast boundary buffer)"), ICA_ERR_NOMEM;
  I.seam_list = fast.seam_list, I.seam_id = fast.seam_id, I.ns = fast.ns;
  I.sflux = (double *)buf("fast_sflux", (size_t)sz.kall * fast.ns * sizeof(double));
  const size_t nsv = (size_t)ntr * sz.kall * fast.ns;
  if (f64) I.sval64 = (double *)buf("fast_sval64", nsv * sizeof(double));
  else I.sval = (float *)buf("fast_sval", nsv * sizeof(float));
  if (!I.sflux || (f64 ? !I.sval64 : !I.sval)) return set_error("cudaMalloc(fast seam buffers)"), ICA_ERR_NOMEM;
  const size_t n3v = (size_t)sz.lall * sz.kall * sz.gall;
  if (f64) {
    I.vco64 = (double4 *)buf("fast_vco64", n3v * sizeof(double4));
    if (!I.vco64) return set_error("cudaMalloc(fast vertical coefficients)"), ICA_ERR_NOMEM;
  } else {
    I.vco = (float4 *)buf("fast_vco", n3v * sizeof(float4));
    if (!I.vco) return set_error("cudaMalloc(fast vertical coefficients)"), ICA_ERR_NOMEM;
  }
  const size_t n3 = (size_t)sz.lall * sz.kall * sz.gall;
  I.Fg = (double *)buf("fast_Fg", 3 * n3 * sizeof(double));
  if (f64) I.dupc64 = (double4 *)buf("fast_dupc64", 3 * n3 * sizeof(double4));
  else I.dupc = (float4 *)buf("fast_dupc", 3 * n3 * sizeof(float4));
  if (!I.Fg || (f64 ? !I.dupc64 : !I.dupc)) return set_error("cudaMalloc(fast face fluxes)"), ICA_ERR_NOMEM;
  if (!fast.err) {  // the device status word, zero until a bounded wait gives up
    fast.err = (int *)buf("fast_err", sizeof(int));
    if (!fast.err || cudaMemsetAsync(fast.err, 0, sizeof(int), stream) != cudaSuccess)
      return set_error("cudaMalloc(fast status word)"), ICA_ERR_NOMEM;
  }
  I.err = fast.err;
  I.work_next = (unsigned long long *)buf("fast_work_next", sizeof(unsigned long long));
  if (!I.work_next) return set_error("cudaMalloc(fast work counter)"), ICA_ERR_NOMEM;
  I.l0 = fast.sharded ? fast.l0 : 0;
  I.l1 = fast.sharded ? fast.l1 : sz.lall;
  I.poles = fast.sharded ? fast.poles : 1;
  return ICA_OK;
}

}  // namespace icoadv

extern "C" {

int ica_fast_shapes(ica_ctx *c, int *n, int *tx, int *ty, int *tg) {
  CTX_OK(c);
  if (!n) return ICA_ERR_ARG;
  *n = fast_tile_shapes(tx, ty, tg, c->sz.gmax - c->sz.gmin + 1);
  return ICA_OK;
}

int ica_fast_set_shape(ica_ctx *c, int shape) {
  CTX_OK(c);
  int n = fast_tile_shapes(nullptr, nullptr, nullptr, 0);
  if (shape < 0 || shape >= n) return set_error("ica_fast_set_shape: no such tile shape"), ICA_ERR_ARG;
  c->fast.shape = shape;
  return ICA_OK;
}

int ica_boundary_tables(int glevel, int rlevel, int *nb, int *bsrc, int *blist, int *pole_ring) {
  if (!nb) return set_error("ica_boundary_tables: NULL count"), ICA_ERR_ARG;
  if (glevel < 1 || rlevel < 0 || rlevel > glevel || glevel > 12)
    return set_error("ica_boundary_tables: bad levels"), ICA_ERR_ARG;
  Topology t(glevel, rlevel);
  std::vector<int> bs, bl, ring;
  const int rc = fast_boundary_tables(t, bs, bl, ring);
  if (rc) return rc;
  *nb = (int)bl.size();
  if (bsrc) std::memcpy(bsrc, bs.data(), bs.size() * sizeof(int));
  if (blist) std::memcpy(blist, bl.data(), bl.size() * sizeof(int));
  if (pole_ring) std::memcpy(pole_ring, ring.data(), ring.size() * sizeof(int));
  return ICA_OK;
}

int ica_fast_status(ica_ctx *c, int *flags) {
  CTX_OK(c);
  if (!flags) return set_error("ica_fast_status: NULL argument"), ICA_ERR_ARG;
  *flags = 0;
  if (!c->fast.err) return ICA_OK;
  cudaSetDevice(c->device);
  cudaError_t e = cudaMemcpyAsync(flags, c->fast.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->fast.err, 0, sizeof(int), c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ica_fast_status");
  return *flags ? ICA_ERR_TIMEOUT : ICA_OK;
}

int ica_fast_set_host_chunk(ica_ctx *c, int tracers) {
  CTX_OK(c);
  if (tracers < 0) return set_error("ica_fast_set_host_chunk: tracers must be >= 0"), ICA_ERR_ARG;
  c->host_chunk = tracers;
  return ICA_OK;
}

int ica_fast_timing(ica_ctx *c, int enable, double *ms_total, long long *count) {
  CTX_OK(c);
  cudaSetDevice(c->device);
  double tot = 0.0;
  long long n = 0;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ica_fast_timing");
  for (auto &p : c->fast.events) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess) tot += ms, ++n;
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  c->fast.events.clear();
  cudaGetLastError();
  c->fast.timing = enable != 0;
  if (ms_total) *ms_total = tot;
  if (count) *count = n;
  return ICA_OK;
}

}  // extern "C"

namespace icoadv {

// fields of one instance: FP32 (float) or FP64 (double, the FP64 variant)
static void set_fields(FastInst &I, const float *vx, const float *vx_pl, const float *vy, const float *vy_pl,
                       const float *vz, const float *vz_pl, const float *w, const float *w_pl) {
  I.vx = vx, I.vy = vy, I.vz = vz, I.w = w, I.vx_pl = vx_pl, I.vy_pl = vy_pl, I.vz_pl = vz_pl, I.w_pl = w_pl;
}
static void set_fields(FastInst &I, const double *vx, const double *vx_pl, const double *vy, const double *vy_pl,
                       const double *vz, const double *vz_pl, const double *w, const double *w_pl) {
  I.vx64 = vx, I.vy64 = vy, I.vz64 = vz, I.w64 = w, I.vx64_pl = vx_pl, I.vy64_pl = vy_pl, I.vz64_pl = vz_pl;
  I.w64_pl = w_pl;
}

template <typename F>
static int advect_fast_impl(Ctx *c, int ntr, double dt, const double *rhog_in, const double *rhog_in_pl,
                            const double *rhogq_in, const double *rhogq_in_pl, double *rhog_out, double *rhog_out_pl,
                            double *rhogq_out, double *rhogq_out_pl, const F *vx, const F *vx_pl, const F *vy,
                            const F *vy_pl, const F *vz, const F *vz_pl, const F *w, const F *w_pl,
                            unsigned parts = 3u) {
  if (ntr < 1 || !rhog_in || !rhog_in_pl || !rhogq_in || !rhogq_in_pl || !rhog_out || !rhog_out_pl || !rhogq_out ||
      !rhogq_out_pl || !vx || !vx_pl || !vy || !vy_pl || !vz || !vz_pl || !w || !w_pl)
    return set_error("ica_advect_fast: NULL argument"), ICA_ERR_ARG;
  if (rhogq_in == rhogq_out || rhog_in == rhog_out)
    return set_error("ica_advect_fast: input and output state must be different buffers"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  FastInst I;
  int rc = c->fast_inst(I, ntr, dt, sizeof(F) == 8);
  if (rc) return rc;
  set_fields(I, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl);
  I.rho_in = rhog_in, I.rho_in_pl = rhog_in_pl, I.Q_in = rhogq_in, I.Q_in_pl = rhogq_in_pl;
  I.rho_out = rhog_out, I.rho_out_pl = rhog_out_pl, I.Q_out = rhogq_out, I.Q_out_pl = rhogq_out_pl;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->fast.timing) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    c->fast.events.push_back({e0, e1});
  }
  cudaError_t e = fast_step(I, c->fast.shape, c->stream, e0, e1, c->launches, parts);
  if (e != cudaSuccess) return cuda_fail(e, "ica_advect_fast");
  if (parts & 2u) {  // the halo fill of the new state (a sharded rank: its own copies only)
    const Plan &p = c->fast.sharded ? c->fast.local : c->plan[0];
    launch_gather<double>(c->D, p.n, p.dst, p.src, c->sz.kall, 1, rhog_out, rhog_out_pl, c->stream);
    launch_gather<double>(c->D, p.n, p.dst, p.src, c->sz.kall, ntr, rhogq_out, rhogq_out_pl, c->stream);
    c->launches += 2;
  }
  return c->check_launch("ica_advect_fast");
}


// Tracers per chunk of the host-pointer step.  The state crosses the host link in chunks: the
// copy of chunk c+1 in and of chunk c-1 out run on their own streams while the step works on
// chunk c, so a step costs about one pass of the state over the link instead of two, plus the
// last chunk's way out.  By size: about 1 GiB of rhogq per chunk, 1 to 4 tracers (four
// tracers are one batch of the horizontal kernel's widest shape).  At glevel 8, kall 96 that
// is 2 tracers: 405 ms per 32-tracer step on a B200 against 424 ms with 1 tracer per chunk and
// 423 ms with 4 (on the same GPU; 384-412 ms for 2 tracers across GPUs).  The copies bound it:
// a chunk's step (about 8 ms for 2 tracers) is shorter than its 23 ms of copies each way.
static int host_chunk_tracers(const Ctx *c, int ntr) {
  if (c->host_chunk > 0) return std::min(ntr, c->host_chunk);
  const size_t per = (size_t)c->sz.gall * c->sz.kall * c->sz.lall * sizeof(double);
  const int t = (int)std::max<size_t>(1, std::min<size_t>(4, ((size_t)1 << 30) / per));
  return std::min(ntr, t);
}

static int advect_fast_chunked(Ctx *c, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq,
                               double *rhogq_pl, const float *vx, const float *vx_pl, const float *vy,
                               const float *vy_pl, const float *vz, const float *vz_pl, const float *w,
                               const float *w_pl) {
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall, n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  const int tc = host_chunk_tracers(c, ntr), nch = (ntr + tc - 1) / tc;
  auto dbl = [&](const char *n, size_t k) { return (double *)c->buf(n, k * sizeof(double)); };
  auto flt = [&](const char *n, size_t k) { return (float *)c->buf(n, k * sizeof(float)); };
  // rho in, rho out (chunk 0; the later chunks recompute the same values into a scratch copy)
  double *r0 = dbl("f0", n3), *r0p = dbl("f1", n3p), *r1 = dbl("f4", n3), *r1p = dbl("f5", n3p);
  double *rs = nch > 1 ? dbl("f8", n3) : r1, *rsp = nch > 1 ? dbl("f9", n3p) : r1p;
  double *qi[2] = {dbl("fq0", n3 * tc), nch > 1 ? dbl("fq1", n3 * tc) : nullptr};
  double *qip[2] = {dbl("fqp0", n3p * tc), nch > 1 ? dbl("fqp1", n3p * tc) : nullptr};
  double *qo[2] = {dbl("fr0", n3 * tc), nch > 1 ? dbl("fr1", n3 * tc) : nullptr};
  double *qop[2] = {dbl("frp0", n3p * tc), nch > 1 ? dbl("frp1", n3p * tc) : nullptr};
  const float *hf[8] = {vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl};
  float *df[8];
  static const char *fname[8] = {"g0", "g1", "g2", "g3", "g4", "g5", "g6", "g7"};
  bool ok = r0 && r0p && r1 && r1p && rs && rsp;
  for (int h = 0; h < (nch > 1 ? 2 : 1); ++h) ok = ok && qi[h] && qip[h] && qo[h] && qop[h];
  for (int v = 0; v < 8; ++v) ok = ok && (df[v] = flt(fname[v], (v & 1) ? n3p : n3)) != nullptr;
  if (!ok) return set_error("ica_advect_fast: cudaMalloc of the staging buffers"), ICA_ERR_NOMEM;

  cudaEvent_t ev[7] = {};  // fields in, chunk in x2, step done x2, chunk out x2
  for (auto &e : ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      for (auto &x : ev)
        if (x) cudaEventDestroy(x);
      return set_error("ica_advect_fast: cudaEventCreate"), ICA_ERR_CUDA;
    }
  cudaEvent_t ev_f = ev[0], *ev_in = ev + 1, *ev_step = ev + 3, *ev_out = ev + 5;
  cudaStream_t sin = c->copy_in, sout = c->copy_out, sc = c->stream;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(cudaMemcpyAsync(r0, rhog, n3 * sizeof(double), cudaMemcpyHostToDevice, sin));
  chk(cudaMemcpyAsync(r0p, rhog_pl, n3p * sizeof(double), cudaMemcpyHostToDevice, sin));
  for (int v = 0; v < 8; ++v)
    chk(cudaMemcpyAsync(df[v], hf[v], ((v & 1) ? n3p : n3) * sizeof(float), cudaMemcpyHostToDevice, sin));
  chk(cudaEventRecord(ev_f, sin));
  chk(cudaStreamWaitEvent(sc, ev_f, 0));
  int rc = ICA_OK;
  for (int ch = 0; ch < nch && e == cudaSuccess && rc == ICA_OK; ++ch) {
    const int b = ch & 1, t0 = ch * tc, nt = std::min(tc, ntr - t0);
    // in: the slot is free once the step of chunk ch-2 has read it
    if (ch >= 2) chk(cudaStreamWaitEvent(sin, ev_step[b], 0));
    chk(cudaMemcpyAsync(qi[b], rhogq + (size_t)t0 * n3, n3 * nt * sizeof(double), cudaMemcpyHostToDevice, sin));
    chk(cudaMemcpyAsync(qip[b], rhogq_pl + (size_t)t0 * n3p, n3p * nt * sizeof(double), cudaMemcpyHostToDevice,
                        sin));
    chk(cudaEventRecord(ev_in[b], sin));
    // step: after its input landed and the output slot of chunk ch-2 went out
    chk(cudaStreamWaitEvent(sc, ev_in[b], 0));
    if (ch >= 2) chk(cudaStreamWaitEvent(sc, ev_out[b], 0));
    if (e != cudaSuccess) break;
    rc = advect_fast_impl<float>(c, nt, dt, r0, r0p, qi[b], qip[b], ch == 0 ? r1 : rs, ch == 0 ? r1p : rsp, qo[b],
                                 qop[b], df[0], df[1], df[2], df[3], df[4], df[5], df[6], df[7]);
    if (rc) break;
    chk(cudaEventRecord(ev_step[b], sc));
    // out
    chk(cudaStreamWaitEvent(sout, ev_step[b], 0));
    if (ch == 0) {
      chk(cudaMemcpyAsync(rhog, r1, n3 * sizeof(double), cudaMemcpyDeviceToHost, sout));
      chk(cudaMemcpyAsync(rhog_pl, r1p, n3p * sizeof(double), cudaMemcpyDeviceToHost, sout));
    }
    chk(cudaMemcpyAsync(rhogq + (size_t)t0 * n3, qo[b], n3 * nt * sizeof(double), cudaMemcpyDeviceToHost, sout));
    chk(cudaMemcpyAsync(rhogq_pl + (size_t)t0 * n3p, qop[b], n3p * nt * sizeof(double), cudaMemcpyDeviceToHost,
                        sout));
    chk(cudaEventRecord(ev_out[b], sout));
  }
  // all three streams drain before the buffers can be reused or the host reads the state
  const cudaError_t s1 = cudaStreamSynchronize(sin), s2 = cudaStreamSynchronize(sc), s3 = cudaStreamSynchronize(sout);
  for (auto &x : ev) cudaEventDestroy(x);
  if (rc) return rc;
  chk(s1), chk(s2), chk(s3);
  if (e != cudaSuccess) return cuda_fail(e, "ica_advect_fast");
  return ICA_OK;
}

}  // namespace icoadv

extern "C" {

int ica_advect_fast_dev(ica_ctx *c, int ntr, double dt, const double *rhog_in, const double *rhog_in_pl,
                        const double *rhogq_in, const double *rhogq_in_pl, double *rhog_out, double *rhog_out_pl,
                        double *rhogq_out, double *rhogq_out_pl, const float *vx, const float *vx_pl, const float *vy,
                        const float *vy_pl, const float *vz, const float *vz_pl, const float *w, const float *w_pl) {
  CTX_OK(c);
  return advect_fast_impl<float>(c, ntr, dt, rhog_in, rhog_in_pl, rhogq_in, rhogq_in_pl, rhog_out, rhog_out_pl,
                                 rhogq_out, rhogq_out_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl);
}

int ica_advect_fast_part_dev(ica_ctx *c, int part, int ntr, double dt, const double *rhog_in,
                             const double *rhog_in_pl, const double *rhogq_in, const double *rhogq_in_pl,
                             double *rhog_out, double *rhog_out_pl, double *rhogq_out, double *rhogq_out_pl,
                             const float *vx, const float *vx_pl, const float *vy, const float *vy_pl, const float *vz,
                             const float *vz_pl, const float *w, const float *w_pl) {
  CTX_OK(c);
  if (part != 1 && part != 2) return set_error("ica_advect_fast_part_dev: part must be 1 or 2"), ICA_ERR_ARG;
  return advect_fast_impl<float>(c, ntr, dt, rhog_in, rhog_in_pl, rhogq_in, rhogq_in_pl, rhog_out, rhog_out_pl,
                                 rhogq_out, rhogq_out_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl,
                                 part == 1 ? 1u : 2u);
}

int ica_shard_set(ica_ctx *c, int l0, int l1, int poles, int nlocal, const int *dst, const int *src) {
  CTX_OK(c);
  int rc = c->need_grid("ica_shard_set");
  if (rc) return rc;
  cudaSetDevice(c->device);
  FastState &f = c->fast;
  if (nlocal < 0) {  // back to the whole grid
    f.sharded = false;
    return ICA_OK;
  }
  const int npt = c->sz.lall * c->sz.gall + kLallPl * kGallPl;
  if (l0 < 0 || l1 > c->sz.lall || l1 <= l0 || (nlocal > 0 && (!dst || !src)))
    return set_error("ica_shard_set: bad region range or copy list"), ICA_ERR_ARG;
  for (int e = 0; e < nlocal; ++e)
    if (dst[e] < 0 || dst[e] >= npt || src[e] < 0 || src[e] >= npt)
      return set_error("ica_shard_set: copy list point out of range"), ICA_ERR_ARG;
  if (f.local.dst) cudaFree(f.local.dst);
  if (f.local.src) cudaFree(f.local.src);
  f.local = Plan{};
  if (cudaMalloc(&f.local.dst, sizeof(int) * (nlocal + 1)) != cudaSuccess ||
      cudaMalloc(&f.local.src, sizeof(int) * (nlocal + 1)) != cudaSuccess)
    return set_error("cudaMalloc(shard copy list)"), ICA_ERR_NOMEM;
  cudaError_t e = cudaMemcpy(f.local.dst, dst, sizeof(int) * nlocal, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(f.local.src, src, sizeof(int) * nlocal, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "ica_shard_set");
  f.local.n = nlocal;
  f.sharded = true;
  f.l0 = l0, f.l1 = l1, f.poles = poles ? 1 : 0;
  return ICA_OK;
}

static int shard_bval(ica_ctx *c, int ntr, int n, const int *bidx, double *buf, bool unpack) {
  CTX_OK(c);
  int rc = c->need_grid("ica_shard_bval");
  if (rc) return rc;
  if (ntr < 1 || n < 0 || (n > 0 && (!bidx || !buf))) return set_error("ica_shard_bval: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  rc = c->build_fast_tables();
  if (rc) return rc;
  double *bbuf = (double *)c->buf("fast_bbuf", (size_t)ntr * c->sz.kall * c->fast.nb * 5 * sizeof(double));
  if (!bbuf) return set_error("cudaMalloc(fast boundary buffer)"), ICA_ERR_NOMEM;
  cudaError_t e = shard_bval_copy(bidx, n, c->fast.nb, c->sz.kall, ntr, bbuf, buf, unpack, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ica_shard_bval");
  c->launches += n > 0;
  return c->check_launch("ica_shard_bval");
}
int ica_shard_bval_pack(ica_ctx *c, int ntr, int n, const int *bidx, double *buf) {
  return shard_bval(c, ntr, n, bidx, buf, false);
}
int ica_shard_bval_unpack(ica_ctx *c, int ntr, int n, const int *bidx, const double *buf) {
  return shard_bval(c, ntr, n, bidx, const_cast<double *>(buf), true);
}

static int shard_points(ica_ctx *c, int n, const int *pts, int kmax, int vmax, double *var, double *var_pl, double *buf,
                        bool unpack) {
  CTX_OK(c);
  if (n < 0 || kmax < 1 || vmax < 1 || (n > 0 && (!pts || !var || !var_pl || !buf)))
    return set_error("ica_shard_points: bad argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  cudaError_t e = shard_point_copy(pts, n, c->sz.lall, c->sz.gall, kmax, vmax, var, var_pl, buf, unpack, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ica_shard_points");
  c->launches += n > 0;
  return c->check_launch("ica_shard_points");
}
int ica_shard_points_pack(ica_ctx *c, int n, const int *pts, int kmax, int vmax, const double *var,
                          const double *var_pl, double *buf) {
  return shard_points(c, n, pts, kmax, vmax, const_cast<double *>(var), const_cast<double *>(var_pl), buf, false);
}
int ica_shard_points_unpack(ica_ctx *c, int n, const int *pts, int kmax, int vmax, double *var, double *var_pl,
                            const double *buf) {
  return shard_points(c, n, pts, kmax, vmax, var, var_pl, const_cast<double *>(buf), true);
}

int ica_advect_fast64_dev(ica_ctx *c, int ntr, double dt, const double *rhog_in, const double *rhog_in_pl,
                          const double *rhogq_in, const double *rhogq_in_pl, double *rhog_out, double *rhog_out_pl,
                          double *rhogq_out, double *rhogq_out_pl, const double *vx, const double *vx_pl,
                          const double *vy, const double *vy_pl, const double *vz, const double *vz_pl,
                          const double *w, const double *w_pl) {
  CTX_OK(c);
  return advect_fast_impl<double>(c, ntr, dt, rhog_in, rhog_in_pl, rhogq_in, rhogq_in_pl, rhog_out, rhog_out_pl,
                                  rhogq_out, rhogq_out_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl);
}

}  // extern "C"

struct ica_batch {
  std::vector<Ctx *> ctx;
  int shape = 0;
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};  // kernel launches a replay of the slot's graph makes
};

namespace icoadv {

template <typename Args>
static int fast_args_ok(const Args &a) {
  return a.ntr >= 1 && a.rhog_in && a.rhog_in_pl && a.rhogq_in && a.rhogq_in_pl && a.rhog_out && a.rhog_out_pl &&
         a.rhogq_out && a.rhogq_out_pl && a.rhogvx && a.rhogvx_pl && a.rhogvy && a.rhogvy_pl && a.rhogvz &&
         a.rhogvz_pl && a.rhogw && a.rhogw_pl && a.rhogq_in != a.rhogq_out && a.rhog_in != a.rhog_out;
}

// instance table of a batch step (device buffers of every instance set up here)
template <typename Args>
static int batch_insts(ica_batch *b, const Args *args, MultiInst &M) {
  constexpr bool f64 = sizeof(*args->rhogvx) == 8;
  M.n = (int)b->ctx.size();
  for (int i = 0; i < M.n; ++i) {
    Ctx *c = b->ctx[i];
    const Args &a = args[i];
    if (!fast_args_ok(a)) return set_error("ica_batch: bad arguments of instance " + std::to_string(i)), ICA_ERR_ARG;
    if (c->fast.sharded) return set_error("ica_batch: instance " + std::to_string(i) + " is a sharded context"), ICA_ERR_STATE;
    c->fast.shape = b->shape;
    FastInst &I = M.inst[i];
    const int rc = c->fast_inst(I, a.ntr, a.dt, f64);
    if (rc) return rc;
    set_fields(I, a.rhogvx, a.rhogvx_pl, a.rhogvy, a.rhogvy_pl, a.rhogvz, a.rhogvz_pl, a.rhogw, a.rhogw_pl);
    I.rho_in = a.rhog_in, I.rho_in_pl = a.rhog_in_pl, I.Q_in = a.rhogq_in, I.Q_in_pl = a.rhogq_in_pl;
    I.rho_out = a.rhog_out, I.rho_out_pl = a.rhog_out_pl, I.Q_out = a.rhogq_out, I.Q_out_pl = a.rhogq_out_pl;
  }
  return ICA_OK;
}

template <typename Args>
static int batch_enqueue(ica_batch *b, const MultiInst &M, const Args *args) {
  Ctx *c0 = b->ctx[0];
  long long launches = 0;
  cudaError_t e = fast_step_multi(M, b->shape, c0->stream, nullptr, nullptr, launches);
  if (e != cudaSuccess) return cuda_fail(e, "ica_batch step");
  for (int i = 0; i < M.n; ++i) {
    Ctx *c = b->ctx[i];
    const Plan &p = c->plan[0];
    launch_gather<double>(c->D, p.n, p.dst, p.src, c->sz.kall, 1, args[i].rhog_out, args[i].rhog_out_pl, c0->stream);
    launch_gather<double>(c->D, p.n, p.dst, p.src, c->sz.kall, args[i].ntr, args[i].rhogq_out, args[i].rhogq_out_pl,
                          c0->stream);
    launches += 2;
  }
  c0->launches += launches;
  return c0->check_launch("ica_batch step");
}

}  // namespace icoadv

extern "C" {

int ica_batch_create(ica_ctx *const *ctxs, int n, ica_batch **out) {
  if (!ctxs || !out || n < 1 || n > ICA_BATCH_MAX) return set_error("ica_batch_create: bad arguments"), ICA_ERR_ARG;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return set_error("ica_batch_create: NULL context"), ICA_ERR_ARG;
    if (ctxs[i]->device != ctxs[0]->device)
      return set_error("ica_batch_create: instances on different devices"), ICA_ERR_ARG;
  }
  ica_batch *b = new ica_batch;
  for (int i = 0; i < n; ++i) b->ctx.push_back(ctxs[i]);
  *out = b;
  return ICA_OK;
}

int ica_batch_destroy(ica_batch *b) {
  if (!b) return ICA_ERR_ARG;
  cudaSetDevice(b->ctx[0]->device);
  for (int s = 0; s < 2; ++s) {
    if (b->exec[s]) cudaGraphExecDestroy(b->exec[s]);
    if (b->graph[s]) cudaGraphDestroy(b->graph[s]);
  }
  delete b;
  return ICA_OK;
}

int ica_batch_set_shape(ica_batch *b, int shape) {
  if (!b) return ICA_ERR_ARG;
  if (shape < 0 || shape >= fast_tile_shapes(nullptr, nullptr, nullptr, 0))
    return set_error("ica_batch_set_shape: no such tile shape"), ICA_ERR_ARG;
  b->shape = shape;
  return ICA_OK;
}

}  // extern "C"

namespace icoadv {

template <typename Args>
static int batch_step_impl(ica_batch *b, const Args *args) {
  if (!b || !args) return set_error("ica_batch_step_dev: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(b->ctx[0]->device);
  MultiInst M;
  int rc = batch_insts(b, args, M);
  if (rc) return rc;
  return batch_enqueue(b, M, args);
}

template <typename Args>
static int batch_capture_impl(ica_batch *b, const Args *args, int slot) {
  if (!b || !args || slot < 0 || slot > 1) return set_error("ica_batch_capture: bad arguments"), ICA_ERR_ARG;
  cudaSetDevice(b->ctx[0]->device);
  MultiInst M;
  int rc = batch_insts(b, args, M);  // every buffer exists before the capture starts
  if (rc) return rc;
  cudaStream_t st = b->ctx[0]->stream;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "ica_batch_capture");
  e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
  long long n0 = 0;
  for (Ctx *c : b->ctx) n0 += c->launches;
  rc = batch_enqueue(b, M, args);
  long long n1 = 0;
  for (Ctx *c : b->ctx) n1 += c->launches;
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  if (b->exec[slot]) cudaGraphExecDestroy(b->exec[slot]);
  if (b->graph[slot]) cudaGraphDestroy(b->graph[slot]);
  b->graph[slot] = g;
  b->exec[slot] = nullptr;
  b->graph_launches[slot] = n1 - n0;
  e = cudaGraphInstantiate(&b->exec[slot], g, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return ICA_OK;
}

}  // namespace icoadv

extern "C" {

int ica_batch_step_dev(ica_batch *b, const ica_fast_args *args) { return batch_step_impl(b, args); }
int ica_batch_step64_dev(ica_batch *b, const ica_fast_args64 *args) { return batch_step_impl(b, args); }
int ica_batch_capture(ica_batch *b, const ica_fast_args *args, int slot) { return batch_capture_impl(b, args, slot); }
int ica_batch_capture64(ica_batch *b, const ica_fast_args64 *args, int slot) {
  return batch_capture_impl(b, args, slot);
}

int ica_batch_replay(ica_batch *b, int slot) {
  if (!b || slot < 0 || slot > 1 || !b->exec[slot]) return set_error("ica_batch_replay: no graph in slot"), ICA_ERR_STATE;
  cudaSetDevice(b->ctx[0]->device);
  cudaError_t e = cudaGraphLaunch(b->exec[slot], b->ctx[0]->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
  b->ctx[0]->launches += b->graph_launches[slot];
  return ICA_OK;
}

int ica_advect_fast(ica_ctx *c, int ntr, double dt, double *rhog, double *rhog_pl, double *rhogq, double *rhogq_pl,
                    const float *vx, const float *vx_pl, const float *vy, const float *vy_pl, const float *vz,
                    const float *vz_pl, const float *w, const float *w_pl) {
  CTX_OK(c);
  if (ntr < 1 || !rhog || !rhog_pl || !rhogq || !rhogq_pl || !vx || !vx_pl || !vy || !vy_pl || !vz || !vz_pl || !w ||
      !w_pl)
    return set_error("ica_advect_fast: NULL argument"), ICA_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = c->copy_streams();
  if (rc) return rc;
  return advect_fast_chunked(c, ntr, dt, rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, w, w_pl);
}

}  // extern "C"
