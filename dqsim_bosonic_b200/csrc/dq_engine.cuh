// dq_engine.cuh — host launchers of the exact per-gate kernels and the
// reduction / sampling kernels (dq_engine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dq_common.cuh"
#include "dq_gates.hpp"

namespace dq {

struct Scratch {            // per-handle device/pinned scratch
  double* d_partial = nullptr;   // kPartials doubles
  unsigned* d_counter = nullptr; // last-block counters
  double* h_pinned = nullptr;    // 64 doubles pinned
  unsigned long long* d_ull = nullptr;
};

constexpr int kPartials = 4096;
constexpr int kRedThreads = 512;

// One classified gate on a state of n qubits.  Returns DQ_OK or an error.
int launch_gate(double2* s, uint32_t n, const GateOp& op, cudaStream_t st, int device,
                uint64_t* launches);

// Number of per-block partial sums the p1 reduction of an n-qubit state uses.
unsigned p1_reduction_blocks(uint32_t n, int device);
// Grid of a reduction kernel over `items` work items (at most kPartials / 4 blocks).
unsigned reduction_blocks(uint64_t items, int device);
// p1 = sum over amplitudes with bit q set (device value in *d_out).
int launch_p1(const double2* s, uint32_t n, uint32_t q, Scratch& sc, double* d_out,
              cudaStream_t st, int device);
// Zero the other half, divide the kept half by norm.
int launch_collapse(double2* s, uint32_t n, uint32_t q, int outcome, double norm,
                    cudaStream_t st, int device);
int launch_set_basis(double2* s, uint32_t n, uint64_t index, cudaStream_t st, int device);

// Device doubles of workspace a marginal over these (physical) qubits needs.
uint64_t marginal_workspace(uint32_t n, const uint32_t* qubits, uint32_t k, int device);
// marginal probabilities into a device buffer d_out[2^k]; d_work holds
// marginal_workspace() doubles (nullptr: a stream-ordered temporary is used).
int launch_marginal(const double2* s, uint32_t n, const uint32_t* qubits, uint32_t k,
                    double* d_out, double* d_work, Scratch& sc, cudaStream_t st, int device);
// Device doubles of workspace launch_cdf needs for len entries.
uint64_t cdf_workspace(uint64_t len);
// in-place inclusive prefix sum of d[len] (deterministic order), last = 1.0;
// d_work holds cdf_workspace(len) doubles (nullptr: a stream-ordered temporary).
int launch_cdf(double* d, uint64_t len, double* d_work, cudaStream_t st, int device);
// per-shot lower_bound in the CDF with device ChaCha8 draws.
int launch_sample(const double* cdf, uint64_t len, const uint32_t key[8], uint64_t shots,
                  uint32_t* d_idx, unsigned long long* d_boundary, cudaStream_t st, int device);

// sum conj(a)*b -> d_out[0..1]; sum |a|^2 -> d_out[0]
int launch_inner(const double2* a, const double2* b, uint32_t n, Scratch& sc, double* d_out,
                 cudaStream_t st, int device);
int launch_norm(const double2* a, uint32_t n, Scratch& sc, double* d_out, cudaStream_t st,
                int device);

}  // namespace dq
