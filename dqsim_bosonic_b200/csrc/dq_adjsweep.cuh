// dq_adjsweep.cuh — fused tile-sweep backward pass of dq_adjoint.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

}  // namespace dq
