// dq_noalloc.cu — the measurement probability p1 without any allocation.
//
// Some callers of this library cannot allocate device memory: hosts that own
// a fixed device-memory budget and hand the library pre-allocated buffers
// only, embedders whose allocator must not be bypassed, and code running in a
// context where cudaMalloc is not permitted.  For them
// dq_measure_p1_noalloc computes p1 = sum of |psi_i|^2 over the amplitudes
// with a given qubit set, for a state vector the caller owns, writing the
// result to a device location the caller owns.  Its only scratch (the
// per-block partial sums and the last-block counter of the reduction) lives
// in the file-scope device array below, which every GPU that loads the
// library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dq_common.cuh"
#include "dq_engine.cuh"

namespace dq {
namespace {

// Room for kNoAllocPartials partial sums followed by the counter word.  The
// p1 reduction launches at most kPartials / 4 blocks (one partial sum each),
// so every n the entry point accepts fits.
constexpr int kNoAllocPartials = 1024;
constexpr size_t kNoAllocScratchBytes = sizeof(double) * kNoAllocPartials + 256;
static_assert(kPartials / 4 <= kNoAllocPartials, "the p1 grid can outgrow the static scratch");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, resolved once per device ordinal and
// kept for the life of the process: a device reset (cudaDeviceReset) or a
// re-created primary context can load the module at another address, after
// which the cached address is stale; do not reset a device this library uses.
std::mutex g_mu;
void* g_addr[64] = {};

int scratch_for_current_device(void** out) {
  int dev = 0;
  DQ_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(DQ_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(DQ_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return DQ_OK;
}

}  // namespace
}  // namespace dq

using namespace dq;

extern "C" {

int dq_measure_p1_noalloc(const double* amps_device, uint32_t n, uint32_t qubit, double* p1_device,
                          void* stream) {
  if (!amps_device || !p1_device) return fail(DQ_ERR_INVALID_ARG, "null device pointer");
  if (n < 1 || n > 34)
    return fail(DQ_ERR_INVALID_ARG, "dq_measure_p1_noalloc: n must be in 1..34");
  if (qubit >= n) return fail(DQ_ERR_INVALID_ARG, "qubit out of range");
  int dev = 0;
  DQ_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned blocks = p1_reduction_blocks(n, dev);
  if (blocks > (unsigned)kNoAllocPartials)
    return fail(DQ_ERR_INVALID_ARG, "dq_measure_p1_noalloc: reduction needs " +
                                        std::to_string(blocks) + " partial sums, the static scratch holds " +
                                        std::to_string(kNoAllocPartials));
  void* base = nullptr;
  DQ_TRY(scratch_for_current_device(&base));
  Scratch sc;
  sc.d_partial = reinterpret_cast<double*>(base);
  sc.d_counter = reinterpret_cast<unsigned*>(reinterpret_cast<unsigned char*>(base) +
                                             sizeof(double) * kNoAllocPartials);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // the last-block counter must start at zero (a previous call leaves it at
  // zero; clearing it here also covers an interrupted call)
  DQ_CUDA_TRY(cudaMemsetAsync(sc.d_counter, 0, sizeof(unsigned), st));
  return launch_p1(reinterpret_cast<const double2*>(amps_device), n, qubit, sc, p1_device, st, dev);
}

}  // extern "C"
