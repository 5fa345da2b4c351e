/*
 * dqsim_cuda.h — C ABI of the B200 (sm_100a) FP64 statevector engine.
 *
 * This header is the drop-in boundary for the statevector hot path of dqsim
 * (Rust crate `dqsim`, module `_core`).  It replaces the free functions of
 * `src/engine.rs` and the per-instruction dispatch of
 * `src/monolithic/statevector/simulator.rs` with calls into a shared library
 * (`libdqsim_cuda.so`) whose state vector stays resident in HBM.
 *
 * Conventions
 *   - Every entry point returns an int status: DQ_OK (0) or a negative
 *     DQ_ERR_* code.  dq_last_error() returns a thread-local message for the
 *     last failing call on the calling thread.  Nothing aborts and no C++
 *     exception crosses this boundary.
 *   - Amplitudes are complex128, stored interleaved (re, im) as double pairs,
 *     index bit q = qubit q (qubit 0 is the least significant bit), exactly the
 *     layout of the reference's `Vec<Complex64>`.
 *   - Gate matrices are row-major complex128 (interleaved), qubits[0] is the
 *     most significant bit of the gate's row/column index (`src/gates.rs`).
 *   - Host buffers are caller-owned; device memory is handle-owned.  Each
 *     handle owns one CUDA stream.  A handle is not thread-safe; distinct
 *     handles may be used concurrently from different threads.
 *   - Calls block until their results are visible to the host.
 *   - No torch types appear in any signature.
 */
#ifndef DQSIM_CUDA_H
#define DQSIM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DQ_ABI_VERSION 1

#if defined(__GNUC__)
#define DQ_API __attribute__((visibility("default")))
#else
#define DQ_API
#endif

/* ---- status codes ------------------------------------------------------ */
#define DQ_OK 0
#define DQ_ERR_INVALID_ARG (-1)    /* bad pointer, size, qubit index ...      */
#define DQ_ERR_CUDA (-2)           /* a CUDA runtime call failed              */
#define DQ_ERR_OOM (-3)            /* device or pinned host allocation failed */
#define DQ_ERR_UNSUPPORTED (-4)    /* unsupported generic gate (NotImplemented) */
#define DQ_ERR_NO_DEVICE (-5)      /* no CUDA device visible                  */
#define DQ_ERR_INTERNAL (-6)       /* invariant violated inside the engine    */
#define DQ_ERR_DECODE (-7)         /* circuit JSON left to the full decoder   */

/* ---- instruction IR ------------------------------------------------------
 * One dq_inst per `Instruction` variant of the reference IR
 * (`src/types.rs:60-135`).  The JSON decoding (serde) stays on the host; the
 * host encodes each decoded instruction into this POD record.
 *
 * Field use per kind (reference field names in brackets):
 *   1q gates            q[0] = qubit
 *   u3/u                p = {theta, phi, lam}
 *   u2                  p = {phi, lam}
 *   u1/p/crz/cu1/cp     p[0] = lam
 *   rx/ry/crx/cry/rxx/rzz p[0] = theta
 *   rz                  p[0] = phi
 *   cu3                 p = {theta, phi, lam};  cu: p = {theta, phi, lam, gamma}
 *   2q controlled       q = {control, target}
 *   swap/rxx/rzz        q = {a, b}
 *   ccx/rccx            q = {control1, control2, target}
 *   cswap               q = {control, target1, target2}
 *   rc3x/c3x/c3sqrtx    q = {control1, control2, control3, target}
 *   c4x                 q = {control1 .. control4, target}
 *   generic gate        q = qubits (nq of them, at most DQ_MAX_INST_QUBITS);
 *                       the host resolves the lower-cased name to a DQ_G_* kind
 *   measure             q[0] = qubit, cbit = cbit
 *   reset               q[0] = qubit
 *   conditional         the wrapped instruction carries cond_count > 0
 *                       conditions starting at conds[cond_first]; nested
 *                       conditionals are flattened (all must hold).
 * ------------------------------------------------------------------------ */
enum dq_kind {
  DQ_ID = 0, DQ_X, DQ_Y, DQ_Z, DQ_H, DQ_S, DQ_SDG, DQ_T, DQ_TDG, DQ_SX, DQ_SXDG,
  DQ_U3, DQ_U2, DQ_U1, DQ_U, DQ_P, DQ_RX, DQ_RY, DQ_RZ, DQ_U0,
  DQ_CX, DQ_CZ, DQ_CY, DQ_CH, DQ_SWAP, DQ_CSX,
  DQ_CRX, DQ_CRY, DQ_CRZ, DQ_CU1, DQ_CP, DQ_CU3, DQ_CU, DQ_RXX, DQ_RZZ,
  DQ_CCX, DQ_CSWAP, DQ_RCCX, DQ_RC3X, DQ_C3X, DQ_C3SQRTX, DQ_C4X,
  /* generic `gate` instructions, resolved by lower-cased name */
  DQ_G_PHI_PLUS,     /* remote_link_phi_plus, remote_epr */
  DQ_G_PSI_MINUS,    /* remote_link_psi_minus */
  DQ_G_PSI_PLUS,     /* remote_link_psi_plus */
  DQ_G_CZ,           /* nonlocal_cz, remote_cz */
  DQ_G_CX,           /* remote_cx */
  DQ_G_NOOP,         /* remote_barrier, remote_cu1 */
  DQ_G_OPAQUE,       /* circuit-*: no-op in the shots path, unsupported in simulate */
  DQ_G_UNSUPPORTED,  /* any other name: DQ_ERR_UNSUPPORTED when executed */
  DQ_MEASURE, DQ_RESET, DQ_BARRIER, DQ_CLASSICAL,
  DQ_KIND_COUNT
};

#define DQ_MAX_INST_QUBITS 8
#define DQ_MAX_GATE_QUBITS 5   /* c4x: the widest gate the engine applies */

typedef struct dq_inst {
  int32_t kind;                      /* enum dq_kind                        */
  int32_t nq;                        /* number of valid entries in q[]      */
  int32_t q[DQ_MAX_INST_QUBITS];     /* qubits in reference field order     */
  int64_t cbit;                      /* measure: target classical bit       */
  double p[4];                       /* parameters in reference field order */
  uint32_t cond_first;               /* index of first condition            */
  uint32_t cond_count;               /* 0 = unconditional                   */
} dq_inst;

typedef struct dq_cond {             /* `Condition` (src/types.rs:54-58)    */
  uint64_t creg_base;
  uint64_t creg_size;                /* <= 64                               */
  uint64_t creg_value;
} dq_cond;

/* ---- circuit JSON decoding ------------------------------------------------
 * Replaces the serde decoding of `circuit.model_dump_json()` into the
 * reference's `Circuit` (src/types.rs:8-135, called from
 * statevector/simulator.rs:327-329) together with the host encoding into
 * dq_inst / dq_cond records.  dq_circuit_decode takes the well-formed case;
 * it returns DQ_ERR_DECODE for invalid JSON, a shape serde rejects, an encoder
 * limit (qubit index >= 2^31, classical space > 2^26 bits, conditions wider
 * than 64 bits, a two-qubit remote gate without two qubits) and a few rare
 * legal forms (duplicate keys, lone surrogate escapes, non-ASCII gate names,
 * numbers that under- or overflow), so that the caller's full decoder reports
 * the exact error or result.  On DQ_OK, dq_circuit_export copies out
 * info->ninst records, info->ncond conditions and info->names_bytes bytes of
 * generic gate names ((uint64 instruction index, uint64 length, bytes)
 * records, names lower-cased); dq_circuit_free releases the object. */
typedef struct dq_circuit dq_circuit;
typedef struct dq_circuit_info {
  uint64_t ninst;
  uint64_t ncond;
  uint64_t num_qubits;   /* max(base + size) over qregs (types.rs:24-31)     */
  uint64_t num_cbits;    /* max(base + size) over cregs (types.rs:33-38)     */
  uint64_t cbit_space;   /* classical bits the run needs (>= 1, <= 2^26)     */
  uint64_t names_bytes;
} dq_circuit_info;

/* ---- options and profile ------------------------------------------------ */
enum dq_semantics {
  DQ_SEM_SIMULATE = 0,  /* run_instruction (simulate):  circuit-* unsupported */
  DQ_SEM_SHOTS = 1      /* run_instruction_par + fuse_circuit (simulate_shots) */
};

enum dq_exec {
  DQ_EXEC_PER_GATE = 0, /* one exact-arithmetic kernel per instruction        */
  DQ_EXEC_FUSED = 1     /* gate runs fused into shared-memory tile sweeps     */
};

typedef struct dq_run_opts {
  int32_t semantics;        /* enum dq_semantics                             */
  int32_t exec;             /* enum dq_exec                                  */
  int32_t fusion_width;     /* local qubits per fused tile; 0 = engine default */
  int32_t profile;          /* nonzero: time each kernel class (per-gate exec) */
  int32_t time_sweeps;      /* nonzero: CUDA-event timing of every fused sweep */
  int32_t max_cost;         /* FP64 ops per amplitude per sweep; 0 = default   */
} dq_run_opts;

typedef struct dq_profile {         /* SimulationProfile (simulator.rs:53-68) */
  uint64_t apply_one_qubit_calls;
  double apply_one_qubit_time;      /* seconds */
  uint64_t apply_n_qubit_calls;
  double apply_n_qubit_time;
  uint64_t measure_qubit_calls;
  double measure_qubit_time;
  double total_time;
  uint64_t kernel_launches;         /* engine kernels launched by the call    */
  uint64_t sweeps;                  /* fused tile sweeps (DQ_EXEC_FUSED)      */
  double sweep_time;                /* seconds in sweeps (time_sweeps != 0)   */
  uint64_t boundary_draws;          /* measure draws with |r - p1| < 1e-12   */
  int64_t failed_inst;              /* index of the failing instruction or -1 */
} dq_profile;

typedef struct dq_state_s* dq_state_t;

/* ---- library ------------------------------------------------------------ */
DQ_API int dq_abi_version(void);
DQ_API const char* dq_last_error(void);
DQ_API int dq_device_count(int* count);

DQ_API int dq_circuit_decode(const char* json, uint64_t len, dq_circuit** out,
                             dq_circuit_info* info);
DQ_API int dq_circuit_export(const dq_circuit* c, dq_inst* insts, dq_cond* conds, uint8_t* names);
DQ_API void dq_circuit_free(dq_circuit* c);

/* ---- state lifecycle ----------------------------------------------------
 * Replaces `vec![C::new(0.0, 0.0); 1 << n]; state[0] = 1`
 * (statevector/simulator.rs:337-339) with an HBM allocation. */
DQ_API int dq_state_create(uint32_t n, int device, dq_state_t* out);
DQ_API int dq_state_destroy(dq_state_t h);
DQ_API int dq_state_num_qubits(dq_state_t h, uint32_t* n);
DQ_API int dq_state_reset(dq_state_t h);                         /* |0...0>          */
DQ_API int dq_state_set_basis(dq_state_t h, uint64_t index);     /* |index>          */
DQ_API int dq_state_upload(dq_state_t h, const double* amps, uint64_t len);   /* len = 2^n */
DQ_API int dq_state_download(dq_state_t h, double* amps, uint64_t len);
DQ_API int dq_state_copy(dq_state_t dst, dq_state_t src);
DQ_API int dq_state_device_ptr(dq_state_t h, void** dev_ptr, void** stream);
DQ_API int dq_state_synchronize(dq_state_t h);

/* ---- gate primitives ----------------------------------------------------
 * dq_apply_1q replaces engine::apply_one_qubit (src/engine.rs:24-101):
 * (psi[i], psi[i|2^t]) <- U (psi[i], psi[i|2^t]) for every i with bit t clear
 * and (i & ctrl_mask) == ctrl_val.  u = {u00, u01, u10, u11} interleaved.   */
DQ_API int dq_apply_1q(dq_state_t h, const double* u, uint32_t target, uint64_t ctrl_mask,
                uint64_t ctrl_val);
/* dq_apply_dense replaces engine::apply_n_qubit (src/engine.rs:109-181):
 * dense 2^k x 2^k (k <= 5) on arbitrary distinct qubits, qubits[0] = MSB.   */
DQ_API int dq_apply_dense(dq_state_t h, const double* u, const uint32_t* qubits, uint32_t k);
/* dq_apply_inst applies one IR instruction exactly as run_instruction
 * (statevector/simulator.rs:386-632) would; measure/reset/conditional are
 * rejected here (use dq_run). */
DQ_API int dq_apply_inst(dq_state_t h, const dq_inst* inst);

/* ---- measurement ---------------------------------------------------------
 * engine::measure_qubit (src/engine.rs:193-257) split at the draw:
 * p1 = sum |psi_i|^2 over bit q set; the caller draws r; outcome = r < p1;
 * the collapse zeroes the other half and divides the kept half by
 * sqrt(p1).max(1e-15) (outcome 1) or sqrt((1-p1).max(0)).max(1e-15).   */
DQ_API int dq_measure_p1(dq_state_t h, uint32_t qubit, double* p1);
DQ_API int dq_collapse(dq_state_t h, uint32_t qubit, int outcome, double p1);
DQ_API int dq_measure(dq_state_t h, uint32_t qubit, double r, int* outcome, double* p1);

/* dq_measure_p1_noalloc: the p1 reduction of dq_measure_p1 for callers that
 * cannot allocate device memory (hosts that own a fixed device-memory
 * budget, embedders whose allocator must not be bypassed, code running where
 * cudaMalloc is not permitted).  No counterpart in the reference: the Rust
 * engine's measure_qubit sums on the CPU and has no device memory to manage.
 * amps_device: a caller-owned device array of 2^n interleaved complex128
 * amplitudes on the current device; p1_device: caller-owned device double
 * that receives p1.  The call only enqueues work on `stream` (a
 * cudaStream_t, NULL = default stream) and returns; it allocates nothing.
 * Its scratch is a static device array of 1024 partial sums (8 KiB + a
 * counter) that every GPU loading the library keeps until exit; the p1
 * reduction never needs more than 1024 of them.  n is limited to 1..34, the
 * engine's largest state (2^34 amplitudes = 256 GiB), and requests needing
 * more partial sums than the array holds are rejected.  The first call on a
 * device resolves the array's address on that device and keeps it for the
 * process (a device reset makes it stale), so make that first call before
 * any stream capture.  All calls share the one array: calls that overlap on
 * the GPU (other streams, other threads) race. */
DQ_API int dq_measure_p1_noalloc(const double* amps_device, uint32_t n, uint32_t qubit,
                                 double* p1_device, void* stream);

/* ---- whole program --------------------------------------------------------
 * Replaces the instruction loop of StatevectorSimulator::simulate
 * (statevector/simulator.rs:351-356) and, with DQ_SEM_SHOTS, one shot of the
 * simulate_shots loop (statevector/simulator.rs:277-285).  The state must
 * hold num_qubits = n.  Outcomes are drawn from ChaCha8Rng::seed_from_u64(seed)
 * in program order, one f64 per executed measure/reset.  cbits[ncbits] is
 * caller-initialised (use -1 for "never written"); measure writes 0/1. */
DQ_API int dq_run(dq_state_t h, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
           uint64_t nconds, uint64_t seed, int32_t* cbits, uint64_t ncbits,
           const dq_run_opts* opts, dq_profile* prof);

/* ---- queries --------------------------------------------------------------
 * engine::marginal_probs (src/engine.rs:368-390): out[j] for j < 2^k,
 * qubits[0] = MSB of j.  k <= n, k <= 30 for this call.                    */
DQ_API int dq_marginal_probs(dq_state_t h, const uint32_t* qubits, uint32_t k, double* out);
/* engine::sample_counts (src/engine.rs:398-433) with the CDF built on the
 * device: out_idx[s] = partition_point(cdf < r_s).min(2^k - 1), r_s the s-th
 * f64 of ChaCha8Rng::seed_from_u64(seed).  *n_boundary counts draws with
 * |r_s - cdf boundary| <= 1e-12 (outcome may differ from a sequential CDF). */
DQ_API int dq_sample(dq_state_t h, const uint32_t* qubits, uint32_t k, uint64_t seed,
              uint64_t shots, uint32_t* out_idx, uint64_t* n_boundary);
/* Same as dq_sample with the 32-byte ChaCha8 key given directly (the
 * reference's from_entropy() path seeds the full key). */
DQ_API int dq_sample_key(dq_state_t h, const uint32_t* qubits, uint32_t k, const uint32_t* key8,
                  uint64_t shots, uint32_t* out_idx, uint64_t* n_boundary);
/* SimulationResult::fidelity inner product <self|other> (simulator.rs:184-191). */
DQ_API int dq_inner(dq_state_t h, const double* other, uint64_t len, double* re, double* im);
DQ_API int dq_norm_sqr(dq_state_t h, double* out);

/* ---- batched shot trajectories ----------------------------------------------
 * simulate_shots (statevector/simulator.rs:216-322) for states of up to 16
 * qubits in one persistent launch: each trajectory (shot s, seed
 * base_seed + shot0 + s, wrapping) runs the fused shot program
 * (types.rs:248-293, run_instruction_par 638-864) on a state held in the
 * shared memory of a thread-block cluster (2^local_bits amplitudes per CTA).
 * cbits_out[s * ncbits + b] receives the shot's classical bits (-1 = never
 * written).  Outcomes match the per-shot dq_run (DQ_SEM_SHOTS) except for
 * draws within 1e-12 of p1, counted in boundary_draws.  ncbits <= 1024. */
typedef struct dq_traj_opts {
  int32_t threads;     /* threads per CTA: 128, 256 or 512 (0 = 256) */
  int32_t max_cluster; /* most CTAs per trajectory: 1, 2, 4 or 8 (0 = 8) */
  int32_t local_bits;  /* amplitudes per CTA = 2^local_bits, 1..13 (0 = min(n, 13)) */
  int32_t reserved;
} dq_traj_opts;

typedef struct dq_traj_stats {
  uint64_t boundary_draws;
  int64_t failed_inst;   /* -1, or the instruction that failed (unsupported gate);
                            dq_run_batch: item << 40 | instruction */
  double kernel_ms;      /* device time of the resident launches (CUDA events) */
  double prepare_ms;     /* host time fusing and encoding the programs */
  double engine_ms;      /* dq_run_batch: host time of items run on the HBM engine */
  uint32_t cluster_span; /* CTAs per trajectory (largest used) */
  uint32_t clusters;     /* clusters resident in the last launch */
  uint32_t threads;
  uint32_t local_bits;   /* amplitudes per CTA = 2^local_bits (largest used) */
  uint32_t launches;     /* persistent launches (plus relabeling passes of HBM items' outputs) */
  uint32_t engine_items; /* dq_run_batch: items run one dq_run each (n > 16 with measurements,
                            resets or conditions) */
  uint32_t hbm_items;    /* dq_run_batch: unitary items of 17..30 qubits run inside the
                            persistent launch as HBM-resident fused sweeps */
  uint32_t reserved;
} dq_traj_stats;

DQ_API int dq_run_trajectories(int device, uint32_t n, const dq_inst* prog, uint64_t ninst,
                               const dq_cond* conds, uint64_t nconds, uint64_t base_seed,
                               uint64_t shot0, uint64_t shots, int32_t* cbits_out,
                               uint64_t ncbits, const dq_traj_opts* opts, dq_traj_stats* stats);

/* The same batch captured once as a CUDA graph (seed upload, counter reset,
 * the persistent launch and the result copies) and replayed per call with a
 * new base seed: shot s of a replay uses seed base_seed + s.  kernel_ms in
 * the stats is the device time of the whole replay. */
typedef struct dq_traj_plan_s* dq_traj_plan_t;
DQ_API int dq_traj_plan_create(int device, uint32_t n, const dq_inst* prog, uint64_t ninst,
                               const dq_cond* conds, uint64_t nconds, uint64_t shots,
                               uint64_t ncbits, const dq_traj_opts* opts, dq_traj_plan_t* out);
DQ_API int dq_traj_plan_run(dq_traj_plan_t plan, uint64_t base_seed, int32_t* cbits_out,
                            dq_traj_stats* stats);
DQ_API int dq_traj_plan_destroy(dq_traj_plan_t plan);

/* A ragged batch of independent circuits, each one trajectory of the shot
 * semantics above (the per-shot loop of statevector/simulator.rs:249-296
 * over circuits of uneven size), in ONE persistent launch taken costliest
 * first from a device work queue: items of up to 16 qubits keep their state
 * in the shared memory of a thread-block cluster; unitary items of 17..30
 * qubits keep it in HBM and run as fused tile sweeps (the planner of the
 * fused engine, 2^11-amplitude tiles) by the CTAs of one cluster, with a
 * cluster barrier between sweeps.  All items share the widest cluster span
 * any of them needs.  Outside that launch: items whose shared-memory slice
 * at that span would hold fewer than 16 amplitudes and, with a forced
 * local_bits, every resident item (launches per cluster span), and large
 * items with measurements, resets or conditions (the HBM engine, dq_run with
 * DQ_SEM_SHOTS, one after another).  Outputs go to the caller's host
 * buffers: the classical bits and, when state_out is non-NULL, the final 2^n
 * complex128 amplitudes. */
typedef struct dq_batch_item {
  uint32_t n;
  uint32_t reserved;
  const dq_inst* prog;
  uint64_t ninst;
  const dq_cond* conds;
  uint64_t nconds;
  uint64_t seed;          /* ChaCha8Rng::seed_from_u64(seed) for its outcomes */
  int32_t* cbits_out;     /* ncbits entries, or NULL when ncbits == 0 */
  uint64_t ncbits;
  double* state_out;      /* 2^n interleaved complex128, or NULL */
} dq_batch_item;

DQ_API int dq_run_batch(int device, const dq_batch_item* items, uint64_t nitems,
                        const dq_traj_opts* opts, dq_traj_stats* stats);

/* ---- observables and adjoint differentiation --------------------------------
 * No counterpart in the reference engine (it has no gradients); the
 * observable convention matches its state layout (qubit q = bit q).
 * A Pauli term is coeff * P with P = prod over qubits q of X_q^x(q) Z_q^z(q)
 * where x(q), z(q) are bits of xmask, zmask, except that a qubit with both
 * bits set carries Y_q = i X_q Z_q.  coeff is real: sum_t terms is Hermitian. */
typedef struct dq_pauli_term {
  double coeff;
  uint64_t xmask; /* qubits carrying X or Y */
  uint64_t zmask; /* qubits carrying Z or Y */
} dq_pauli_term;

/* <psi|H|psi> of the handle's state for H = sum of terms (nterms <= 65536). */
DQ_API int dq_expval_pauli(dq_state_t h, const dq_pauli_term* terms, uint64_t nterms, double* out);

/* Adjoint gradient of E = <psi|H|psi>, psi = U_prog |psi0>, where psi0 is the
 * state the handle holds on entry.  prog must be unitary: gates only, no
 * measure/reset/conditions (barrier/id are skipped).  param_index[4*i + j] is
 * the entry of grad[nparams] that parameter p[j] of instruction i feeds
 * (-1 = held fixed); grad receives the sum over all slots feeding an entry.
 * Differentiable kinds: rx ry rz p u1 u2 u3 u crx cry crz cp cu1 cu3 cu rxx rzz;
 * a slot of any other kind must be -1.  opts selects the forward pass
 * (DQ_EXEC_FUSED or DQ_EXEC_PER_GATE; semantics must be DQ_SEM_SIMULATE).
 * The backward pass walks the program in reverse, uncomputing psi with the
 * inverse gates alongside lambda = H psi (no stored intermediate states; one
 * extra state-sized buffer).  On return the handle holds psi0 again, up to
 * rounding.  param_index may be NULL when nparams == 0 (E only).  phase_ms,
 * when non-NULL, receives 4 values: the device time (ms) of the forward pass,
 * of lambda = H psi and of the backward pass, then the number of fused
 * backward sweeps (0 with DQ_EXEC_PER_GATE). */
DQ_API int dq_adjoint(dq_state_t h, const dq_inst* prog, uint64_t ninst,
                      const int32_t* param_index, uint64_t nparams,
                      const dq_pauli_term* terms, uint64_t nterms,
                      const dq_run_opts* opts, double* expval, double* grad,
                      double* phase_ms);

/* Adjoint gradients of nsets parameter sets of one circuit at once (no
 * counterpart in the reference, which has no gradients).  Set s runs `prog`
 * from |0...0> on `nqubits` qubits with every parameter slot that
 * param_index maps to p (param_index as in dq_adjoint) replaced by
 * values[s * nparams + p]; its E_s goes to expvals[s] and
 * dE_s/d(value p) to grads[s * nparams + p].  The sets share each launch:
 * every fused forward sweep, lambda = H psi, and every fused backward sweep
 * runs for all sets at once (one launch per sweep index; the sets' tiles are
 * (set, chunk) work items), with the states of as many sets as fit in about
 * half of the free device memory resident at a time.  Programs the batched
 * sweeps cannot represent (gates of three or more qubits without a sweep
 * form, fewer than 10 qubits) run set by set through dq_adjoint;
 * stats->batched tells which path ran. */
typedef struct dq_adjoint_batch_stats {
  uint64_t launches;         /* kernel launches of the batched path */
  uint64_t forward_sweeps;   /* sweep indices of the forward pass (largest set) */
  uint64_t backward_sweeps;  /* sweep indices of the backward pass (largest set) */
  double plan_ms;            /* host planning of all sets */
  double forward_ms;         /* device time, all groups */
  double observable_ms;
  double backward_ms;
  uint32_t batched;          /* 1: batched launches; 0: set by set */
  uint32_t groups;           /* groups of sets resident at a time */
} dq_adjoint_batch_stats;

DQ_API int dq_adjoint_batch(int device, uint32_t nqubits, const dq_inst* prog, uint64_t ninst,
                            const int32_t* param_index, uint64_t nparams, const double* values,
                            uint64_t nsets, const dq_pauli_term* terms, uint64_t nterms,
                            double* expvals, double* grads, dq_adjoint_batch_stats* stats);

/* ---- p-block merge -----------------------------------------------------------
 * merge_blocks (src/distributed/pblock/model.rs:35-57): the tensor product of
 * block a (state of the ascending qubits a_qubits[0..na)) and block b into
 * `out`, whose qubits are the ascending union of both lists (a qubit named in
 * both takes one position).  out must have exactly that many qubits and be a
 * third state; it is overwritten.  Amplitude i of out is a[la(i)] * b[lb(i)]
 * with num-complex's multiplication (no FMA): bit-identical to the
 * reference.  All three states must live on one device. */
DQ_API int dq_block_merge(dq_state_t a, const uint32_t* a_qubits, uint32_t na, dq_state_t b,
                          const uint32_t* b_qubits, uint32_t nb, dq_state_t out);

/* ---- matrix-product-state backend -----------------------------------------
 * MpsSimulator (src/monolithic/mps/simulator.rs:293-455): one MPS per handle
 * (dq_mps_create, max_bond = 0 for max_bond_dimension=None) or a batch of
 * independent shots (dq_mps_run_shots).  dq_mps_run replaces the instruction
 * loop of MpsSimulator::simulate (:316-344): the state restarts at |0...0>,
 * the outcomes draw from ChaCha8Rng::seed_from_u64(seed), cbits as in dq_run.
 * Two-qubit gates are chains of fused adjacent steps (contract, SVD, keep the
 * singular values above truncation_threshold, at least 1, at most max_bond,
 * renormalise: apply_adjacent_2q :137-236).  dq_mps_to_state writes
 * to_statevector (:238-257) into a statevector handle of n qubits.
 * dq_mps_run_shots replaces the shot loop of MpsSimulator::simulate_shots
 * (:368-385): shot i is seeded base_seed + shot0 + i (wrapping), its cbits
 * go to row i of cbits_out (shots x ncbits, -1 = never written); batch = 0
 * picks the replicas per launch.  DQ_ERR_UNSUPPORTED (stats->failed_inst =
 * the instruction) for gates on three or more qubits and unknown generic
 * names, raised when such an instruction executes (:540-557). */
typedef struct dq_mps_s* dq_mps_t;
typedef struct dq_mps_stats {
  uint64_t svd_calls;     /* two-qubit SVD steps executed, over all replicas */
  double kernel_ms;       /* device time of the program's launches */
  int64_t failed_inst;    /* DQ_ERR_UNSUPPORTED: index of the instruction */
  uint32_t capacity;      /* bond-dimension capacity the run ended with */
  uint32_t replicas;      /* replicas per launch */
} dq_mps_stats;
DQ_API int dq_mps_create(uint32_t n, int device, uint32_t max_bond, double truncation_threshold,
                         dq_mps_t* out);
DQ_API int dq_mps_destroy(dq_mps_t h);
DQ_API int dq_mps_run(dq_mps_t h, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
                      uint64_t nconds, uint64_t seed, int32_t* cbits, uint64_t ncbits,
                      dq_mps_stats* stats);
/* Mps::apply_2q (:115-135) on the current state: u = 4x4 row-major complex
 * (interleaved re/im, 32 doubles), a = most significant qubit of the row.
 * A step that needs a wider bond capacity widens the handle (dq_mps_reserve)
 * and redoes the step; if that allocation fails the call returns DQ_ERR_OOM
 * with the swap-chain steps done so far applied and the handle still usable. */
DQ_API int dq_mps_apply_2q(dq_mps_t h, uint32_t a, uint32_t b, const double* u);
/* Widen the bond capacity of a single-state handle, keeping its state, bond
 * dimensions and RNG position (its classical bits are not kept: a later
 * dq_mps_run starts them afresh).  If the wider buffers cannot be allocated
 * the state is put back at the old capacity and the allocation error is
 * returned; only if that also fails is the handle left unusable (every later
 * call on it fails; destroy it). */
DQ_API int dq_mps_reserve(dq_mps_t h, uint32_t capacity);
DQ_API int dq_mps_bond_dims(dq_mps_t h, uint32_t* dims);   /* n + 1 entries */
DQ_API int dq_mps_to_state(dq_mps_t h, dq_state_t out);
DQ_API int dq_mps_run_shots(int device, uint32_t n, uint32_t max_bond, double truncation_threshold,
                            const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
                            uint64_t nconds, uint64_t base_seed, uint64_t shot0, uint64_t shots,
                            int32_t* cbits_out, uint64_t ncbits, uint32_t batch,
                            dq_mps_stats* stats);

/* ---- planner inspection (host only, no GPU needed) -------------------------
 * Runs the fused-sweep planner of dq_run (DQ_EXEC_FUSED) on a unitary
 * program of n qubits and writes the encoded sweep programs instead of
 * launching them.  out receives: u32 magic 0x4C505144 ("DQPL"), u32 nsweeps,
 * u32 register bits, u32 0, u32 perm[64] (logical -> physical after the
 * program), u64 offset[nsweeps] into the blob, then the blob.  *len is the
 * byte count needed (call with cap = 0 to size the buffer). */
DQ_API int dq_debug_plan(uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_run_opts* opts,
                         uint8_t* out, uint64_t cap, uint64_t* len);

/* ---- RNG (host side; same stream the device uses) ------------------------
 * ChaCha8Rng::seed_from_u64(seed) (rand_chacha 0.3.1 / rand_core 0.6.4),
 * gen::<f64>() (rand 0.8.5): the draws at positions [skip, skip + count). */
DQ_API int dq_rng_f64(uint64_t seed, uint64_t skip, uint64_t count, double* out);
DQ_API int dq_rng_seed_key(uint64_t seed, uint32_t* key8);
DQ_API int dq_chacha_block(const uint32_t* in16, uint32_t rounds, uint32_t* out16);

#ifdef __cplusplus
}
#endif
#endif /* DQSIM_CUDA_H */
