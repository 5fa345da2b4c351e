// dq_reduce.cuh — deterministic block and grid reductions shared by the
// engine's reduction kernels (p1, norm, inner products, observables and
// adjoint gradients).
#pragma once

#include <cuda_runtime.h>

namespace dq {
namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the block; the result is valid in thread 0.  Fixed tree order.
__device__ double block_sum(double v) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// Writes this block's partial(s); the last block to finish sums all partials
// in index order (deterministic for a fixed grid) into out[0..W).
template <int W>
__device__ void finish_partials(const double (&v)[W], double* partial, unsigned* counter,
                                double* out) {
  __shared__ bool last;
  double tot[W];
#pragma unroll
  for (int c = 0; c < W; ++c) tot[c] = block_sum(v[c]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < W; ++c) partial[c * gridDim.x + blockIdx.x] = tot[c];
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int c = 0; c < W; ++c) {
    double a = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
      a = __dadd_rn(a, __ldcg(partial + c * gridDim.x + i));
    a = block_sum(a);
    if (threadIdx.x == 0) out[c] = a;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace
}  // namespace dq
