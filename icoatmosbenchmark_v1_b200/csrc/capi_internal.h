// Context object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "icoadv_internal.h"
#include "plain_kernels.cuh"
#include "step.cuh"

namespace icoadv {

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};

struct Plan {  // composed halo fill on the device
  int n = 0;
  int *dst = nullptr, *src = nullptr;
};

struct FastState {  // fused path: boundary tables, tile shape, kernel timing
  bool built = false;
  int nb = 0, shape = 0;
  int *bsrc = nullptr, *blist = nullptr, *ring = nullptr, *carry = nullptr;
  int *seam_list = nullptr, *seam_id = nullptr;
  int ncarry = 0, ns = 0;
  float *cg32 = nullptr;
  float *off32 = nullptr;  // per-face remap offsets, rebuilt when the geometry changes
  bool off_ready = false;
  double *off64 = nullptr;  // the same in FP64 (FP64 variant)
  bool off64_ready = false;
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  int *err = nullptr;  // device status word of the batched kernels (a buffer of the context)
  // region-sharded run (ica_shard_set): this context computes regions [l0, l1) and, with
  // poles, the pole centres; `local` holds the halo copies whose two points it owns
  bool sharded = false;
  int l0 = 0, l1 = 0, poles = 1;
  Plan local;
};

struct FastInst;

struct AdjTape {  // a recorded multi-step run: checkpoints every `every` steps
  bool ready = false;
  int ntr = 0, nsteps = 0, every = 0;
  double dt = 0.0;
};

struct Ctx {
  std::unique_ptr<Topology> topo;
  ica_sizes sz{};
  Dims D{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;  // host-link copies of the chunked host path
  int host_chunk = 0;                                   // tracers per chunk of that path, 0: by size
  Plan plan[2];               // [0] COMM_data_transfer, [1] COMM_var
  int *d_have_sgp = nullptr;
  void *geo64[8] = {};        // GRD_xr, _pl, GMTR_p, _pl, GMTR_t, _pl, GMTR_a, _pl
  void *geo32[8] = {};
  std::vector<size_t> geo_n;
  bool geo_set = false;
  void *stepgeo[7] = {};      // GRD_x, GRD_x_pl, coef_grad, coef_grad_pl, rdgz, afact, bfact
  bool stepgeo_set = false;
  std::map<std::string, DevBuf> bufs;  // staging / scratch, grow-only
  long long launches = 0;

  ~Ctx();
  // contexts made by ica_init_regions hold part of a grid (the arrays a reference driver
  // holds) and no region topology: what needs the whole grid returns ICA_ERR_STATE
  int need_grid(const char *what) const;
  void *buf(const char *name, size_t bytes);
  void release(const char *name);
  int check_launch(const char *what);
  int copy_streams();
  int upload_geometry(const double *const h[8], const size_t n[8]);
  template <typename T> Geo<T> geo() const;
  int step_ctx(StepCtx &S);
  FastState fast;
  int build_fast_tables();
  int fast_inst(FastInst &I, int ntr, double dt, bool f64 = false);
  AdjTape tape;
  // device address of the fixed scratch of ica_horizontal_limiter_thuburn_noalloc on this
  // context's device, looked up by ica_init (nullptr if that lookup failed)
  double *noalloc_scratch = nullptr;
};

int cuda_fail(cudaError_t e, const char *what);

// horizontal_limiter_thuburn on device buffers with caller-provided scratch: the Qout copy
// the halo fill runs on (gall*kall*lall*2 and 6*kall*2*2 values) and the pole inflow bounds
// (6*kall*2*4 values).  Instantiated for double in capi.cu.
template <typename T>
int hlim_dev(Ctx *c, T *q_a, T *q_a_pl, const T *q, const T *q_pl, const T *d, const T *d_pl, const T *ch,
             const T *ch_pl, const T *cmask, const T *cmask_pl, T *Qout_prev, T *Qout_prev_pl, const T *Qout_post,
             const T *Qout_post_pl, T *scratch_Qout, T *scratch_Qout_pl, T *scratch_Qin_pl);

// Device address of the noalloc limiter's fixed scratch array in the current device's
// context.  Looking it up loads the module that holds the array, so its device memory is
// taken at that moment (ica_init calls this).
int noalloc_scratch_address(double **out);

}  // namespace icoadv
