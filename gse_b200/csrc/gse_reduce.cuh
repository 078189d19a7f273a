// gse_reduce.cuh -- deterministic block and grid reductions of doubles shared
// by the energy kernels (gse_kernels.cu, gse_fft.cu).
#pragma once

#include "gse_internal.cuh"

namespace gse {

// ---------------------------------------------------------------------------
// Block reduction of a double into partials[blockIdx.x] (fixed order).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_sum_to(double v, double* partials) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double s = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) partials[blockIdx.x] = s;
  }
}

// After block_sum_to: the block that finishes last (a counter in
// partials[gridDim.x], zero between launches) adds the partials in index
// order -- the result does not depend on which block ran when -- and writes
// factor * sum to out[0].
__device__ __forceinline__ void last_block_sum_counter(double* partials, unsigned* done,
                                                       double factor, double* out);
__device__ __forceinline__ void last_block_sum(double* partials, double factor, double* out) {
  last_block_sum_counter(partials, reinterpret_cast<unsigned*>(partials + gridDim.x), factor,
                         out);
}
// As last_block_sum with the counter at `done`.
__device__ __forceinline__ void last_block_sum_counter(double* partials, unsigned* done,
                                                       double factor, double* out) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;  // uniform in the block
  __threadfence();
  __shared__ double red[32];
  double t = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
    t += ((volatile double*)partials)[i];
  t = warp_sum(t);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = t;
  __syncthreads();
  if (w == 0) {
    double u = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    u = warp_sum(u);
    if (lane == 0) {
      out[0] = u * factor;
      *done = 0u;
    }
  }
}

}  // namespace gse
