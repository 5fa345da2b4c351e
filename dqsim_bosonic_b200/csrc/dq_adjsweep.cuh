// dq_adjsweep.cuh — fused tile-sweep backward pass of dq_adjoint.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/dqsim_cuda.h"

namespace dq {

struct AdjSweepStats {
  uint64_t sweeps = 0;   // fused sweeps launched
  uint64_t pergate = 0;  // gates undone one at a time (three or more qubits)
};

// Walks prog in reverse on psi (holding U psi0) and lambda (holding H U psi0),
// undoing every gate on both and writing the gradient term of every active
// parameter slot (program order, as numbered by param_index) to d_slots
// (without the factor 2).
int adjoint_backward_fused(double2* psi, double2* lam, uint32_t n, const dq_inst* prog,
                           uint64_t ninst, const int32_t* param_index, uint64_t nslots,
                           double* d_slots, cudaStream_t st, int device, AdjSweepStats* stats);

// One parameter set's backward pass encoded as fused sweeps (host memory):
// sweep k has header record k, op records from op0[k], slot map entries
// from slot0[k] (nslots[k] of them); matrices index into `pool`.
struct ABatchSet {
  std::vector<uint8_t> hdrs;  // sweep header records, one per sweep
  std::vector<uint8_t> ops;   // op records of all sweeps
  std::vector<double2> pool;
  std::vector<uint32_t> map;
  std::vector<size_t> op0, slot0;  // per sweep: first op record, first map entry
  std::vector<uint32_t> nslots;
  size_t sweeps() const { return nslots.size(); }
};

// Plans the backward pass of one parameter set; DQ_ERR_UNSUPPORTED when a
// gate of three or more qubits needs the per-gate kernels.
int adjoint_backward_plan_set(uint32_t n, const dq_inst* prog, uint64_t ninst,
                              const int32_t* param_index, uint64_t nslots, ABatchSet* out);

// The backward pass of B parameter sets (set b: psi[b], lam[b] on the device,
// gradient slots written to d_slots[b]): sweep k of every set in one launch
// (plus one slot reduction launch); counts launches.
int adjoint_backward_batch(double2* const* psi, double2* const* lam,
                           const std::vector<ABatchSet>& sets, double* const* d_slots,
                           cudaStream_t st, int device, uint64_t* launches);

}  // namespace dq
