// dq_fused.cuh — fused tile-sweep execution of gate programs.
//
// A unitary stretch of the program (between measurements) is planned into
// "sweeps".  Each sweep streams the state through HBM once: a CTA stages a
// tile of 2^m amplitudes (the m "local" qubits: qubits 0..4 plus up to m-5
// chosen ones) in shared memory, applies every gate of the sweep whose
// non-diagonal action stays on local qubits, and writes the tile back.
// Diagonal gates of degree <= 2 (z, s, t, p, rz, cz, cp, crz, rzz, ...) are
// kept as a pending phase polynomial and applied lazily right before the
// first non-diagonal gate on one of their qubits, whether that qubit is
// local or not.  swap gates relabel qubits (no data movement); the final
// relabeling is undone by the store of the last sweep.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <vector>

#include "dq_common.cuh"
#include "dq_gates.hpp"

namespace dq {

struct FusedWork {
  // plan-only mode (no GPU work): encoded sweep programs are appended here
  std::vector<uint8_t>* plan_out = nullptr;
  std::vector<uint64_t>* plan_offs = nullptr;
  uint32_t plan_rb = 0;
  // plan-only mode: thread bits of the kernel that will run the programs (0:
  // the default launch geometry); out: the basis index the first planned sweep
  // generates its tiles from (-1: it reads the state)
  uint32_t plan_tb = 0;
  int64_t plan_synth = -1;
  uint8_t* d_blob = nullptr;
  size_t d_cap = 0;
  uint8_t* h_blob = nullptr;  // pinned staging
  size_t h_cap = 0;
  std::vector<cudaEvent_t> events;
};

void fused_release(FusedWork& fw);

struct FusedHooks {
  // p1 + draw + collapse on a physical qubit (the host RNG cursor lives in the caller)
  std::function<int(uint32_t phys_q, int* outcome)> measure;
  // exact per-gate kernel on physical qubits (reset's X, gates the planner cannot fuse)
  std::function<int(const GateOp& op)> exact_gate;
  int32_t* cbits = nullptr;
  uint64_t ncbits = 0;
  const dq_cond* conds = nullptr;
  // the state's pending basis index (>= 0: memory not yet written): the first
  // sweep synthesises its tiles from it and clears it
  int64_t* lazy_basis = nullptr;
};

// perm[l] = physical position of logical qubit l; updated in place (swap
// gates relabel instead of moving data).
int fused_run(double2* amp, uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_run_opts& o,
              FusedWork& fw, cudaStream_t st, int device, FusedHooks& hooks, dq_profile* prof,
              uint32_t* perm);

// Move the data so that perm becomes the identity (two paired-tile sweeps at
// most); sets perm[l] = l.
int materialize_perm(double2* amp, uint32_t n, uint32_t* perm, cudaStream_t st,
                     uint64_t* launches);

// Smallest register width the fused path runs (smaller states use per-gate kernels).
constexpr uint32_t kFusedMinQubits = 10;

// Plans a unitary program as fused sweeps without running anything: the
// encoded programs are appended to *blob (their offsets to *offs), *rb is
// the register bits of the geometry, perm is updated by the swaps, and
// *synth receives the basis index the first sweep generates its tiles from
// (lazy_basis >= 0: the program starts from that basis vector) or -1.
// tb = 0: the default thread geometry; fusion_width 0: the default tile.
int fused_plan(uint32_t n, const dq_inst* prog, uint64_t ninst, int semantics, uint32_t tb,
               int fusion_width, int64_t lazy_basis, std::vector<uint8_t>* blob,
               std::vector<uint64_t>* offs, uint32_t* perm, int64_t* synth, uint32_t* rb);

// One sweep of one state in a multi-state launch.
struct SweepJob {
  double2* state;
  const uint8_t* prog;  // device pointer to an encoded sweep program
  long long synth;      // >= 0: generate the input from this basis index
  uint32_t prog_bytes, pad;
};

// Runs one sweep of each of njobs states (all of n qubits, programs planned
// with 7 thread bits, register width rb and the same run width run_bits, none
// longer than max_bytes) in ONE launch; d_jobs is device memory.  flags: the
// AND of the programs' header flags (sweep_flags), which selects a restricted
// kernel build when every program allows it.
int launch_sweep_multi(const SweepJob* d_jobs, uint32_t njobs, uint32_t n, uint32_t rb,
                       uint32_t run_bits, uint32_t max_bytes, cudaStream_t st, uint32_t flags);

// The run width (5 or 3) and the size of an encoded sweep program in host memory.
uint32_t sweep_run_bits(const uint8_t* prog);
uint32_t sweep_prog_bytes(const uint8_t* prog);
// The kernel-choice flags of an encoded sweep program in host memory.
uint32_t sweep_flags(const uint8_t* prog);

}  // namespace dq
