// Launch interface of the batched path.
#pragma once

#include <cuda_runtime.h>

#include "fast_common.cuh"

namespace icoadv {

// Tile shapes available to the autotuner: fills tx/ty/tg (arrays of the returned length) when non-NULL.
int fast_tile_shapes(int *tx, int *ty, int *tg, int nmax);
// Per-face remap offsets (GRD_xr - GRD_x of the owner and of the neighbour, FP32) into
// off (lall, 18, gall); needs I's geometry pointers only.
cudaError_t fast_build_offsets(const FastInst &I, float *off, cudaStream_t st);
cudaError_t fast_build_offsets64(const FastInst &I, double *off, cudaStream_t st);  // the same in FP64
// One step of instance I on stream st with tile shape `shape` (of k_fast_horiz); ev0/ev1
// (optional) are recorded around k_fast_horiz, the dominant launch.
// parts: bit 0 the boundary pass, bit 1 the rest of the step (a region-sharded run exchanges
// the boundary values between the two).
cudaError_t fast_step(const FastInst &I, int shape, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                      long long &launches, unsigned parts = 3u);
// The same step for M.n grid instances (uneven grid levels) together, all of one precision
// (FastInst::f64: the FP32 or the FP64 variant): each kernel is one
// launch over the work of every instance; the horizontal kernel is persistent (one wave of
// CTAs striding over all (instance, level, tile) items).  Launches nothing that allocates,
// so it can be captured in a CUDA graph once every instance has run one step uncaptured.
cudaError_t fast_step_multi(const MultiInst &M, int shape, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                            long long &launches, unsigned parts = 3u);
// Region-sharded runs: copy the boundary values of the indices bidx[n] between the context's
// boundary buffer (ntr, K, nb, 5) and buf (ntr, K, n, 5), or points pts[n] of a region array
// (vmax, lall, kmax, gall) with its pole array (vmax, 2, kmax, 6) and buf (vmax, kmax, n);
// unpack = buf -> array.
cudaError_t shard_bval_copy(const int *bidx, int n, int nb, int K, int ntr, double *bbuf, double *buf, bool unpack,
                            cudaStream_t st);
cudaError_t shard_point_copy(const int *pts, int n, int lall, int gall, int kmax, int vmax, double *var,
                             double *var_pl, double *buf, bool unpack, cudaStream_t st);

}  // namespace icoadv
