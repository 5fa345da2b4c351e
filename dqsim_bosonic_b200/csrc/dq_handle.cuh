// dq_handle.cuh — the state handle behind dq_state_t and the helpers the
// extern "C" translation units (dq_api.cu, dq_adjoint.cu) share.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_fused.cuh"
#include "dq_gates.hpp"

struct dq_state_s {
  int device = 0;
  uint32_t n = 0;
  uint64_t len = 0;
  size_t bytes = 0;
  double2* amp = nullptr;
  cudaStream_t stream = nullptr;
  dq::Scratch sc;
  dq::FusedWork fw;
  // perm[l] = physical bit position holding logical qubit l (fused runs
  // relabel swap gates instead of moving data)
  uint32_t perm[64];
  bool permuted = false;
  // >= 0: the state is the physical basis vector |lazy_basis> but memory has
  // not been written yet; the next fused sweep synthesises its input tiles
  // from it (no read of the state, no reset pass), anything else writes it
  // first (materialize_basis)
  int64_t lazy_basis = -1;
  // query buffers (marginals, CDF, sampled indices): kept and grown as needed
  // so that a query allocates nothing per call
  void* q_dev = nullptr;
  size_t q_dev_cap = 0;
  void* q_host = nullptr;  // pinned
  size_t q_host_cap = 0;
};

namespace dq {

constexpr uint32_t kMaxQubits = 34;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Device buffers of state size are recycled through a per-(device, size) cache.
int cache_alloc(int device, size_t bytes, void** out);
void cache_free(int device, size_t bytes, void* p);
// Pinned host staging buffers (at least `bytes`), recycled by size class.
int pinned_alloc(size_t bytes, void** out);
void pinned_free(size_t bytes, void* p);

int check_handle(dq_state_t h);            // validates and materialises a lazy basis state
int check_handle_lazy(dq_state_t h);       // validates only
int materialize_basis(dq_state_t h);
int sync_stream(dq_state_t h);
// Make the physical layout canonical (undo a pending qubit relabeling).
int canonicalize(dq_state_t h);
// Mark the layout canonical without moving data (the state is rewritten).
void reset_perm(dq_state_t h);
// Copy `count` device doubles to `out` through the handle's pinned buffer.
int read_scalars(dq_state_t h, const double* d_src, int count, double* out);
// Grow the handle's query buffers to at least dev_bytes (device) and
// host_bytes (pinned host); the stream is drained before a buffer is replaced.
int ensure_query_buffers(dq_state_t h, size_t dev_bytes, size_t host_bytes);
int gate_qubit_count(int kind);
int validate_inst(const dq_inst& in, uint32_t n, uint64_t nconds, uint64_t ncbits,
                  const dq_cond* conds, uint64_t idx);
// Reduce a gate instruction to its kernel class (false: no matrix).
bool inst_to_op(const dq_inst& in, GateOp& op);

}  // namespace dq
