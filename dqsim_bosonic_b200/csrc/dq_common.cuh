// dq_common.cuh — shared helpers of the dqsim B200 engine.
//
// Complex128 arithmetic in the exact operation order of num-complex 0.4.6
// (mul = (ar*br - ai*bi, ar*bi + ai*br), no fused multiply-add), so the
// per-gate kernels reproduce src/engine.rs bit for bit.  The fused sweep
// kernels use the FMA variants (cmul_fma) and are held to a tolerance.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/dqsim_cuda.h"

namespace dq {

// ---- error plumbing --------------------------------------------------------
void set_error(const std::string& msg);
void clear_error();

struct Status {
  int code;
};

#define DQ_CUDA_TRY(expr)                                                       \
  do {                                                                          \
    cudaError_t e__ = (expr);                                                   \
    if (e__ != cudaSuccess) {                                                   \
      ::dq::set_error(std::string(#expr) + ": " + cudaGetErrorString(e__));     \
      return (e__ == cudaErrorMemoryAllocation) ? DQ_ERR_OOM : DQ_ERR_CUDA;     \
    }                                                                           \
  } while (0)

#define DQ_TRY(expr)             \
  do {                           \
    int rc__ = (expr);           \
    if (rc__ != DQ_OK) return rc__; \
  } while (0)

inline int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

// ---- exact complex arithmetic (device) ------------------------------------
__device__ __forceinline__ double2 cmul_x(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cadd_x(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double norm_sqr_x(double2 a) {
  return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
}

// ---- fused-multiply-add complex arithmetic (device) ------------------------
__device__ __forceinline__ double2 cmul_f(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a*x + b*y
__device__ __forceinline__ double2 cmac2_f(double2 a, double2 x, double2 b, double2 y) {
  double re = fma(a.x, x.x, fma(-a.y, x.y, fma(b.x, y.x, -b.y * y.y)));
  double im = fma(a.x, x.y, fma(a.y, x.x, fma(b.x, y.y, b.y * y.x)));
  return make_double2(re, im);
}

// ---- index helpers ---------------------------------------------------------
// Insert a zero bit at each position of the ascending list pos[0..np).
__host__ __device__ __forceinline__ uint64_t insert_zeros(uint64_t k, const uint32_t* pos,
                                                          int np) {
  for (int i = 0; i < np; ++i) {
    const uint32_t p = pos[i];
    k = ((k >> p) << (p + 1)) | (k & ((1ULL << p) - 1ULL));
  }
  return k;
}

__host__ __device__ __forceinline__ uint64_t insert_zero(uint64_t k, uint32_t p) {
  return ((k >> p) << (p + 1)) | (k & ((1ULL << p) - 1ULL));
}

// Stream-ordered allocation from the engine's per-device memory pool on the
// current device (free with cudaFreeAsync); the pool keeps freed memory for
// the next call instead of returning it at every synchronisation.
cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t st);

// Grid sizing: blocks for `work` items, capped at a multiple of the SM count.
unsigned grid_for(uint64_t work, unsigned threads, int device);

}  // namespace dq
