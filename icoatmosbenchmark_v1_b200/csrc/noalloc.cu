// horizontal_limiter_thuburn for callers that cannot allocate device memory.
//
// The ordinary entry points take their scratch (the copy of Qout that the
// halo fill runs on, and the pole-ring inflow bounds) from buffers the
// context allocates with cudaMalloc on first use.  Some callers cannot let a
// library do that: a host model that hands the whole GPU to its own pool
// allocator at start-up and allocates every array exactly once (the usual
// shape of a Fortran climate model), or a run whose device-memory footprint
// must not change once it has started.  For them this file keeps the scratch
// in a fixed-size array in the library's own device memory: every GPU that
// loads the library holds it (16.6 MiB) until the process exits, and this
// entry point calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits: gall*kall*lall <= ICA_NOALLOC_MAX_CELLS and kall <= ICA_NOALLOC_MAX_KALL;
// larger grids are rejected with ICA_ERR_ARG.  All calls share the one array:
// calls that overlap on the GPU (other streams, other threads) race.
#include <cuda_runtime.h>

#include <mutex>

#include "capi_internal.h"

namespace icoadv {

constexpr size_t kRegionScratch = (size_t)2 * ICA_NOALLOC_MAX_CELLS;        // Qout copy, 2 values per cell
constexpr size_t kPoleQout = (size_t)kGallPl * kLallPl * 2 * ICA_NOALLOC_MAX_KALL;  // Qout_pl copy
constexpr size_t kPoleQin = (size_t)kGallPl * kLallPl * 4 * ICA_NOALLOC_MAX_KALL;   // Qin_pl(min/max, face set)

static __device__ __align__(256) double g_noalloc_scratch[kRegionScratch + kPoleQout + kPoleQin];

// Device address of g_noalloc_scratch on `device`, looked up once per device
// (the host-side symbol is only a stand-in, never a device address).
static int noalloc_scratch(int device, double **out) {
  static std::mutex mu;
  static double *addr[64] = {};
  if (device < 0 || device >= 64) return set_error("noalloc: device ordinal out of range"), ICA_ERR_ARG;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    addr[device] = (double *)p;
  }
  *out = addr[device];
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
  if (!q_a || !q_a_pl || !q || !q_pl || !d || !d_pl || !ch || !ch_pl || !cmask || !cmask_pl || !Qout_prev ||
      !Qout_prev_pl || ((Qout_post == nullptr) != (Qout_post_pl == nullptr)))
    return set_error("ica_horizontal_limiter_thuburn_noalloc: bad argument"), ICA_ERR_ARG;
  const size_t n3 = (size_t)c->sz.gall * c->sz.kall * c->sz.lall;
  if (n3 > (size_t)ICA_NOALLOC_MAX_CELLS || c->sz.kall > ICA_NOALLOC_MAX_KALL)
    return set_error("ica_horizontal_limiter_thuburn_noalloc: grid exceeds the fixed scratch "
                     "(gall*kall*lall <= ICA_NOALLOC_MAX_CELLS, kall <= ICA_NOALLOC_MAX_KALL)"),
           ICA_ERR_ARG;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  double *scratch = nullptr;
  int rc = noalloc_scratch(c->device, &scratch);
  if (rc) return rc;
  double *s_qout = scratch, *s_qout_pl = scratch + kRegionScratch, *s_qin_pl = scratch + kRegionScratch + kPoleQout;
  const size_t n3p = (size_t)kGallPl * c->sz.kall * kLallPl;
  LimIn<double> in{q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl};
  // Qout before the fill; the pole kernel writes every Qin_pl element the apply reads
  launch_hlim_qout<double>(c->D, in, Qout_prev, Qout_prev_pl, s_qin_pl, c->stream);
  c->launches += 2;
  const double *Qo = Qout_post, *Qo_pl = Qout_post_pl;
  if (!Qout_post) {  // the halo fill on a copy of Qout (every element of the copy is overwritten)
    cudaMemcpyAsync(s_qout, Qout_prev, n3 * 2 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(s_qout_pl, Qout_prev_pl, n3p * 2 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    const Plan &p = c->plan[0];
    launch_gather<double>(c->D, p.n, p.dst, p.src, c->sz.kall, 2, s_qout, s_qout_pl, c->stream);
    c->launches += 1;
    Qo = s_qout;
    Qo_pl = s_qout_pl;
  }
  launch_hlim_apply<double>(c->D, in, q_a, q_a_pl, Qo, Qo_pl, s_qin_pl, c->stream);
  c->launches += 2;
  return c->check_launch("ica_horizontal_limiter_thuburn_noalloc");
}
