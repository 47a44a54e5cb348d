// horizontal_limiter_thuburn for callers that cannot allocate device memory.
//
// The ordinary entry points take their scratch (the copy of Qout that the
// halo fill runs on, and the pole-ring inflow bounds) from buffers the
// context allocates with cudaMalloc on first use.  Some callers cannot let a
// library do that: a host model that hands the whole GPU to its own pool
// allocator at start-up and allocates every array exactly once (the usual
// shape of a Fortran climate model), or a run whose device-memory footprint
// must not change once it has started.  For them this file keeps the scratch
// in a fixed-size array in the library's own device memory (about 32.1 MiB):
// ica_init looks up its address, which loads it on the context's device, so
// the context must be created before the host's pool claims the GPU.  From then
// on every GPU with a context holds the array until the process exits, and
// this entry point calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits: gall*kall*lall <= ICA_NOALLOC_MAX_CELLS and kall <= ICA_NOALLOC_MAX_KALL;
// larger grids are rejected with ICA_ERR_ARG.  All calls share the one array:
// calls that overlap on the GPU (other streams, other threads) race.
#include <cuda_runtime.h>

#include "capi_internal.h"

namespace icoadv {

constexpr size_t kRegionScratch = (size_t)2 * ICA_NOALLOC_MAX_CELLS;        // Qout copy, 2 values per cell
constexpr size_t kPoleQout = (size_t)kGallPl * kLallPl * 2 * ICA_NOALLOC_MAX_KALL;  // Qout_pl copy
constexpr size_t kPoleQin = (size_t)kGallPl * kLallPl * 4 * ICA_NOALLOC_MAX_KALL;   // Qin_pl(min/max, face set)

static __device__ __align__(256) double g_noalloc_scratch[kRegionScratch + kPoleQout + kPoleQin];

// The host-side symbol g_noalloc_scratch is only a stand-in, never a device address:
// the address is looked up in the current device's context.
int noalloc_scratch_address(double **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  *out = (double *)p;
  return ICA_OK;
}

}  // namespace icoadv

using namespace icoadv;

extern "C" int ica_horizontal_limiter_thuburn_noalloc(ica_ctx *ctx, double *q_a, double *q_a_pl, const double *q,
                                                      const double *q_pl, const double *d, const double *d_pl,
                                                      const double *ch, const double *ch_pl, const double *cmask,
                                                      const double *cmask_pl, double *Qout_prev,
                                                      double *Qout_prev_pl, const double *Qout_post,
                                                      const double *Qout_post_pl) {
  if (!ctx) return set_error("NULL context"), ICA_ERR_ARG;
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall;
  if (n3 > (size_t)ICA_NOALLOC_MAX_CELLS || c->sz.kall > ICA_NOALLOC_MAX_KALL)
    return set_error("ica_horizontal_limiter_thuburn_noalloc: grid exceeds the fixed scratch "
                     "(gall*kall*lall <= ICA_NOALLOC_MAX_CELLS, kall <= ICA_NOALLOC_MAX_KALL)"),
           ICA_ERR_ARG;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  if (!c->noalloc_scratch) {  // the lookup at ica_init failed: try once more, report what fails
    int rc = noalloc_scratch_address(&c->noalloc_scratch);
    if (rc) return rc;
  }
  double *s = c->noalloc_scratch;
  return hlim_dev<double>(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl, Qout_prev, Qout_prev_pl,
                          Qout_post, Qout_post_pl, s, s + kRegionScratch, s + kRegionScratch + kPoleQout);
}
