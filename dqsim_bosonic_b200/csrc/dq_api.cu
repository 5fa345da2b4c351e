// dq_api.cu — the extern "C" boundary (include/dqsim_cuda.h): state
// handles, gate primitives, measurement, the program runner and queries.
//
// dq_run is the instruction dispatcher of the reference
// (statevector/simulator.rs:386-632 for simulate, 638-884 + types.rs:248-293
// for one simulate_shots trajectory) moved below the C ABI, so a host that
// keeps the reference's JSON decoding hands over the whole program once and
// the state never leaves HBM.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_fused.cuh"
#include "dq_gates.hpp"
#include "dq_handle.cuh"
#include "dq_rng.cuh"

namespace dq {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
void clear_error() { g_err.clear(); }

// ---- stream-ordered scratch ----------------------------------------------------
// Small per-call device buffers (observable terms, sweep programs of the
// adjoint pass, reduction workspaces) come from one memory pool per device
// that keeps up to 256 MiB when idle: the default pool returns its memory at
// every synchronisation, so the next call would map it again.
cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static cudaMemPool_t pools[64];
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev & 63]) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev & 63], &props);
      if (e != cudaSuccess) {
        pools[dev & 63] = nullptr;
        return e;
      }
      uint64_t keep = 256ull << 20;
      e = cudaMemPoolSetAttribute(pools[dev & 63], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = pools[dev & 63];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

// ---- HBM buffer cache ---------------------------------------------------------
// State vectors are large (16 GiB at 30 qubits); a destroyed state's buffer is
// kept for the next state of the same size on the same device.
namespace {
std::mutex g_cache_mu;
std::map<std::pair<int, size_t>, std::vector<void*>> g_cache;
constexpr size_t kMaxCachedPerKey = 2;
}  // namespace

int cache_alloc(int device, size_t bytes, void** out) {
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find({device, bytes});
    if (it != g_cache.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      return DQ_OK;
    }
  }
  cudaError_t e = cudaMalloc(out, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto& kv : g_cache) {
      if (kv.first.first != device) continue;
      for (void* p : kv.second) cudaFree(p);
      kv.second.clear();
    }
    e = cudaMalloc(out, bytes);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,
                std::string("cudaMalloc(") + std::to_string(bytes) + " B): " +
                    cudaGetErrorString(e));
  }
  return DQ_OK;
}

void cache_free(int device, size_t bytes, void* p) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto& v = g_cache[{device, bytes}];
  if (v.size() < kMaxCachedPerKey) {
    v.push_back(p);
  } else {
    cudaFree(p);
  }
}

// Pinned host staging buffers, kept by size class (a power of two of at
// least 1 MiB) so that repeated large uploads neither page-fault fresh host
// memory nor pay cudaHostAlloc.
std::mutex g_pinned_mu;
std::map<size_t, std::vector<void*>> g_pinned;

size_t pinned_class(size_t bytes) {
  size_t c = 1ULL << 20;
  while (c < bytes) c <<= 1;
  return c;
}

int pinned_alloc(size_t bytes, void** out) {
  const size_t c = pinned_class(bytes);
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    auto it = g_pinned.find(c);
    if (it != g_pinned.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      return DQ_OK;
    }
  }
  cudaError_t e = cudaHostAlloc(out, c, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return fail(DQ_ERR_OOM, std::string("cudaHostAlloc(") + std::to_string(c) + " B): " +
                                cudaGetErrorString(e));
  }
  return DQ_OK;
}

void pinned_free(size_t bytes, void* p) {
  if (!p) return;
  const size_t c = pinned_class(bytes);
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  auto& v = g_pinned[c];
  if (v.size() < kMaxCachedPerKey) {
    v.push_back(p);
  } else {
    cudaFreeHost(p);
  }
}

}  // namespace dq


using namespace dq;

namespace dq {

// ---- handle shells --------------------------------------------------------------
// Up to kMaxShells destroyed handles per device keep their stream, reduction
// scratch, pinned buffer and fused-sweep buffers for the next dq_state_create.
namespace {
std::mutex g_shell_mu;
std::vector<dq_state_t> g_shells[64];
constexpr size_t kMaxShells = 8;
}  // namespace

dq_state_t take_shell(int device) {
  std::lock_guard<std::mutex> lk(g_shell_mu);
  auto& v = g_shells[device & 63];
  if (v.empty()) return nullptr;
  dq_state_t h = v.back();
  v.pop_back();
  return h;
}

bool put_shell(dq_state_t h) {
  std::lock_guard<std::mutex> lk(g_shell_mu);
  auto& v = g_shells[h->device & 63];
  if (v.size() >= kMaxShells) return false;
  v.push_back(h);
  return true;
}

int check_handle_lazy(dq_state_t h) {
  if (!h || !h->amp) return fail(DQ_ERR_INVALID_ARG, "null or destroyed state handle");
  return DQ_OK;
}

int materialize_basis(dq_state_t h) {
  if (h->lazy_basis < 0) return DQ_OK;
  DeviceGuard g(h->device);
  DQ_TRY(launch_set_basis(h->amp, h->n, (uint64_t)h->lazy_basis, h->stream, h->device));
  h->lazy_basis = -1;
  return DQ_OK;
}

int check_handle(dq_state_t h) {
  DQ_TRY(check_handle_lazy(h));
  return materialize_basis(h);
}

int sync_stream(dq_state_t h) {
  DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DQ_OK;
}

// Query outputs up to this size use the handle's kept buffers; larger ones a
// temporary allocation (a 30-qubit marginal alone is 8 GiB).
constexpr size_t kQueryKeepBytes = 64ULL << 20;

// A device buffer for one query: the handle's kept buffer, or a temporary one
// freed (after the stream drains) when the object goes out of scope.
struct QueryBuffer {
  dq_state_t h = nullptr;
  void* tmp = nullptr;
  void* ptr = nullptr;
  ~QueryBuffer() {
    if (tmp) {
      cudaStreamSynchronize(h->stream);
      cudaFree(tmp);
    }
  }
  int get(dq_state_t hh, size_t bytes) {
    h = hh;
    if (bytes <= kQueryKeepBytes) {
      DQ_TRY(ensure_query_buffers(h, bytes, 0));
      ptr = h->q_dev;
      return DQ_OK;
    }
    cudaError_t e = cudaMalloc(&tmp, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      tmp = nullptr;
      return fail(DQ_ERR_OOM, std::string("cudaMalloc(query output): ") + cudaGetErrorString(e));
    }
    ptr = tmp;
    return DQ_OK;
  }
};

int ensure_query_buffers(dq_state_t h, size_t dev_bytes, size_t host_bytes) {
  if (dev_bytes > h->q_dev_cap) {
    DQ_TRY(sync_stream(h));
    if (h->q_dev) cudaFree(h->q_dev);
    h->q_dev = nullptr;
    h->q_dev_cap = 0;
    const size_t cap = std::max<size_t>(dev_bytes, 64 * 1024);
    cudaError_t e = cudaMalloc(&h->q_dev, cap);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(DQ_ERR_OOM, std::string("cudaMalloc(query buffer): ") + cudaGetErrorString(e));
    }
    h->q_dev_cap = cap;
  }
  if (host_bytes > h->q_host_cap) {
    DQ_TRY(sync_stream(h));
    if (h->q_host) cudaFreeHost(h->q_host);
    h->q_host = nullptr;
    h->q_host_cap = 0;
    const size_t cap = std::max<size_t>(host_bytes, 64 * 1024);
    cudaError_t e = cudaMallocHost(&h->q_host, cap);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(DQ_ERR_OOM, std::string("cudaMallocHost(query buffer): ") + cudaGetErrorString(e));
    }
    h->q_host_cap = cap;
  }
  return DQ_OK;
}

void reset_perm(dq_state_t h) {
  for (uint32_t l = 0; l < 64; ++l) h->perm[l] = l;
  h->permuted = false;
}

// Make the physical layout canonical (perm = identity).
int canonicalize(dq_state_t h) {
  DQ_TRY(materialize_basis(h));
  if (!h->permuted) return DQ_OK;
  DQ_TRY(materialize_perm(h->amp, h->n, h->perm, h->stream, nullptr));
  h->permuted = false;
  return DQ_OK;
}

void update_permuted(dq_state_t h) {
  h->permuted = false;
  for (uint32_t l = 0; l < h->n; ++l)
    if (h->perm[l] != l) h->permuted = true;
}

uint64_t map_mask(dq_state_t h, uint64_t mask) {
  uint64_t out = 0;
  for (uint32_t l = 0; l < h->n; ++l)
    if (mask >> l & 1ULL) out |= 1ULL << h->perm[l];
  return out;
}

int read_scalars(dq_state_t h, const double* d_src, int count, double* out) {
  DQ_CUDA_TRY(cudaMemcpyAsync(h->sc.h_pinned, d_src, sizeof(double) * count,
                              cudaMemcpyDeviceToHost, h->stream));
  DQ_TRY(sync_stream(h));
  for (int i = 0; i < count; ++i) out[i] = h->sc.h_pinned[i];
  return DQ_OK;
}

int gate_qubit_count(int kind) {
  if (kind >= DQ_ID && kind <= DQ_U0) return 1;
  if (kind >= DQ_CX && kind <= DQ_RZZ) return 2;
  if (kind >= DQ_CCX && kind <= DQ_RCCX) return 3;
  if (kind >= DQ_RC3X && kind <= DQ_C3SQRTX) return 4;
  if (kind == DQ_C4X) return 5;
  if (kind >= DQ_G_PHI_PLUS && kind <= DQ_G_CX) return 2;
  if (kind == DQ_MEASURE || kind == DQ_RESET) return 1;
  return 0;  // generic no-op / unsupported / barrier / classical
}

int validate_inst(const dq_inst& in, uint32_t n, uint64_t nconds, uint64_t ncbits,
                  const dq_cond* conds, uint64_t idx) {
  auto bad = [&](const std::string& m) {
    return fail(DQ_ERR_INVALID_ARG, "instruction " + std::to_string(idx) + ": " + m);
  };
  if (in.kind < 0 || in.kind >= DQ_KIND_COUNT) return bad("unknown kind");
  if (in.nq < 0 || in.nq > DQ_MAX_INST_QUBITS) return bad("bad qubit count");
  const int need = gate_qubit_count(in.kind);
  if (need > 0) {
    if (in.nq != need)
      return bad("expected " + std::to_string(need) + " qubits, got " + std::to_string(in.nq));
    for (int a = 0; a < need; ++a) {
      if (in.q[a] < 0 || (uint32_t)in.q[a] >= n)
        return bad("qubit index " + std::to_string(in.q[a]) + " out of range for " +
                   std::to_string(n) + " qubits");
      for (int b = 0; b < a; ++b)
        if (in.q[a] == in.q[b]) return bad("repeated qubit " + std::to_string(in.q[a]));
    }
  }
  if (in.kind == DQ_MEASURE && (in.cbit < 0 || (uint64_t)in.cbit >= ncbits))
    return bad("cbit outside the classical register array");
  if (in.cond_count > 0) {
    if (!conds || (uint64_t)in.cond_first + in.cond_count > nconds)
      return bad("condition range outside the condition array");
    for (uint32_t c = 0; c < in.cond_count; ++c)
      if (conds[in.cond_first + c].creg_size > 64) return bad("condition wider than 64 bits");
  }
  return DQ_OK;
}

bool cond_holds(const dq_inst& in, const dq_cond* conds, const int32_t* cbits, uint64_t ncbits) {
  for (uint32_t c = 0; c < in.cond_count; ++c) {
    const dq_cond& cd = conds[in.cond_first + c];
    uint64_t actual = 0;
    for (uint64_t b = 0; b < cd.creg_size; ++b) {
      const uint64_t idx = cd.creg_base + b;
      const uint64_t v = (idx < ncbits && cbits[idx] > 0) ? (uint64_t)cbits[idx] : 0;
      actual |= v << b;
    }
    if (actual != cd.creg_value) return false;
  }
  return true;
}

// Reduce a gate instruction to its kernel class.
bool inst_to_op(const dq_inst& in, GateOp& op) {
  hc u[4];
  if (matrix_1q(in.kind, in.p, u)) {
    classify_1q(u, (uint32_t)in.q[0], 0, op);
    return true;
  }
  Gate g;
  if (!matrix_nq(in, g)) return false;
  classify(g, op);
  return true;
}

// Timing of one kernel class (profile=True): events bracketing the calls.
struct ProfileTimer {
  bool on = false;
  cudaStream_t st = nullptr;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[3];  // oq, nq, mq
  std::vector<cudaEvent_t> pool;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  cudaEvent_t begin() {
    if (!on) return nullptr;
    cudaEvent_t e = get();
    cudaEventRecord(e, st);
    return e;
  }
  void end(int cls, cudaEvent_t b) {
    if (!on) return;
    cudaEvent_t e = get();
    cudaEventRecord(e, st);
    ev[cls].push_back({b, e});
  }
  void collect(dq_profile* p) {
    if (!on || !p) return;
    cudaStreamSynchronize(st);
    double* t[3] = {&p->apply_one_qubit_time, &p->apply_n_qubit_time, &p->measure_qubit_time};
    for (int c = 0; c < 3; ++c)
      for (auto& pr : ev[c]) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        *t[c] += ms * 1e-3;
      }
  }
  ~ProfileTimer() {
    for (int c = 0; c < 3; ++c)
      for (auto& pr : ev[c]) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
      }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

struct RunCtx {
  dq_state_t h;
  Chacha8Cursor rng;
  int32_t* cbits;
  uint64_t ncbits;
  dq_profile prof;
  ProfileTimer timer;
  int sem;
};

int do_measure(RunCtx& c, uint32_t q, int* outcome) {
  dq_state_t h = c.h;
  cudaEvent_t b = c.timer.begin();
  DQ_TRY(launch_p1(h->amp, h->n, q, h->sc, h->sc.d_partial + kPartials - 1, h->stream, h->device));
  double p1 = 0.0;
  DQ_TRY(read_scalars(h, h->sc.d_partial + kPartials - 1, 1, &p1));
  const double r = c.rng.draw();
  const int o = (r < p1) ? 1 : 0;
  if (fabs(r - p1) < 1e-12) ++c.prof.boundary_draws;
  double norm;
  if (o == 1) {
    norm = sqrt(p1);
    if (norm < 1e-15) norm = 1e-15;
  } else {
    double t = 1.0 - p1;
    if (t < 0.0) t = 0.0;
    norm = sqrt(t);
    if (norm < 1e-15) norm = 1e-15;
  }
  DQ_TRY(launch_collapse(h->amp, h->n, q, o, norm, h->stream, h->device));
  c.prof.kernel_launches += 2;
  c.timer.end(2, b);
  ++c.prof.measure_qubit_calls;
  *outcome = o;
  return DQ_OK;
}

int do_gate_op(RunCtx& c, const GateOp& op, int cls) {
  cudaEvent_t b = c.timer.begin();
  DQ_TRY(launch_gate(c.h->amp, c.h->n, op, c.h->stream, c.h->device, &c.prof.kernel_launches));
  c.timer.end(cls, b);
  if (cls == 0) ++c.prof.apply_one_qubit_calls; else ++c.prof.apply_n_qubit_calls;
  return DQ_OK;
}

// One instruction whose conditions hold.
int exec_inst(RunCtx& c, const dq_inst& in) {
  switch (in.kind) {
    case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP:
      return DQ_OK;
    case DQ_G_OPAQUE:
      if (c.sem == DQ_SEM_SHOTS) return DQ_OK;
      return fail(DQ_ERR_UNSUPPORTED, "unsupported generic gate");
    case DQ_G_UNSUPPORTED:
      return fail(DQ_ERR_UNSUPPORTED, "unsupported generic gate");
    case DQ_MEASURE: {
      int o = 0;
      DQ_TRY(do_measure(c, (uint32_t)in.q[0], &o));
      c.cbits[in.cbit] = o;
      return DQ_OK;
    }
    case DQ_RESET: {
      int o = 0;
      DQ_TRY(do_measure(c, (uint32_t)in.q[0], &o));
      if (o == 1) {
        GateOp op;
        hc u[4];
        matrix_1q(DQ_X, nullptr, u);
        classify_1q(u, (uint32_t)in.q[0], 0, op);
        DQ_TRY(do_gate_op(c, op, 0));
      }
      return DQ_OK;
    }
    default:
      break;
  }
  GateOp op;
  if (!inst_to_op(in, op)) return fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
  return do_gate_op(c, op, gate_qubit_count(in.kind) == 1 ? 0 : 1);
}

}  // namespace dq

// =========================================================================
// extern "C"
// =========================================================================
extern "C" {

int dq_abi_version(void) { return DQ_ABI_VERSION; }

const char* dq_last_error(void) { return g_err.c_str(); }

int dq_device_count(int* count) {
  if (!count) return fail(DQ_ERR_INVALID_ARG, "null count");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return fail(DQ_ERR_NO_DEVICE, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = c;
  return DQ_OK;
}

int dq_state_create(uint32_t n, int device, dq_state_t* out) {
  if (!out) return fail(DQ_ERR_INVALID_ARG, "null output handle");
  *out = nullptr;
  if (n > kMaxQubits)
    return fail(DQ_ERR_INVALID_ARG, "num_qubits " + std::to_string(n) + " exceeds the engine limit of " +
                                        std::to_string(kMaxQubits));
  int ndev = 0;
  DQ_TRY(dq_device_count(&ndev));
  if (ndev == 0) return fail(DQ_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(DQ_ERR_INVALID_ARG, "device index out of range");
  DeviceGuard g(device);
  // a destroyed handle's shell (stream, scratch, pinned buffer, sweep program
  // buffers) is reused: creating those costs milliseconds per simulate call
  if (dq_state_t sh = take_shell(device)) {
    sh->n = n;
    sh->len = 1ULL << n;
    sh->bytes = sizeof(double2) * sh->len;
    void* p = nullptr;
    const int rc = cache_alloc(device, sh->bytes, &p);
    if (rc != DQ_OK) {
      put_shell(sh);
      return rc;
    }
    sh->amp = (double2*)p;
    reset_perm(sh);
    sh->lazy_basis = 0;  // |0...0>, written by the first sweep or on first use
    *out = sh;
    return DQ_OK;
  }
  dq_state_t h = new (std::nothrow) dq_state_s();
  if (!h) return fail(DQ_ERR_OOM, "host allocation failed");
  h->device = device;
  h->n = n;
  h->len = 1ULL << n;
  h->bytes = sizeof(double2) * h->len;
  void* p = nullptr;
  int rc = cache_alloc(device, h->bytes, &p);
  if (rc != DQ_OK) {
    delete h;
    return rc;
  }
  h->amp = (double2*)p;
  reset_perm(h);
  auto cleanup = [&](int code, const char* what, cudaError_t e) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    cudaGetLastError();
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->sc.d_partial) cudaFree(h->sc.d_partial);
    if (h->sc.d_counter) cudaFree(h->sc.d_counter);
    if (h->sc.h_pinned) cudaFreeHost(h->sc.h_pinned);
    cache_free(device, h->bytes, h->amp);
    delete h;
    return code;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cleanup(DQ_ERR_CUDA, "cudaStreamCreate", e);
  e = cudaMalloc((void**)&h->sc.d_partial, sizeof(double) * kPartials);
  if (e != cudaSuccess) return cleanup(DQ_ERR_OOM, "cudaMalloc(scratch)", e);
  e = cudaMalloc((void**)&h->sc.d_counter, sizeof(unsigned) * 16 + sizeof(unsigned long long) * 8);
  if (e != cudaSuccess) return cleanup(DQ_ERR_OOM, "cudaMalloc(counters)", e);
  h->sc.d_ull = (unsigned long long*)(h->sc.d_counter + 16);
  e = cudaMemsetAsync(h->sc.d_counter, 0, sizeof(unsigned) * 16 + sizeof(unsigned long long) * 8,
                      h->stream);
  if (e != cudaSuccess) return cleanup(DQ_ERR_CUDA, "cudaMemset(counters)", e);
  e = cudaMallocHost((void**)&h->sc.h_pinned, sizeof(double) * 64);
  if (e != cudaSuccess) return cleanup(DQ_ERR_OOM, "cudaMallocHost", e);
  rc = sync_stream(h);
  if (rc != DQ_OK) {
    dq_state_destroy(h);
    return rc;
  }
  h->lazy_basis = 0;  // |0...0>, written by the first sweep or on first use
  *out = h;
  return DQ_OK;
}

int dq_state_destroy(dq_state_t h) {
  if (!h) return DQ_OK;
  DeviceGuard g(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->amp) cache_free(h->device, h->bytes, h->amp);
  h->amp = nullptr;
  if (h->stream && h->sc.d_partial && h->sc.d_counter && h->sc.h_pinned && put_shell(h))
    return DQ_OK;
  fused_release(h->fw);
  if (h->q_dev) cudaFree(h->q_dev);
  if (h->q_host) cudaFreeHost(h->q_host);
  if (h->sc.d_partial) cudaFree(h->sc.d_partial);
  if (h->sc.d_counter) cudaFree(h->sc.d_counter);
  if (h->sc.h_pinned) cudaFreeHost(h->sc.h_pinned);
  if (h->stream) cudaStreamDestroy(h->stream);
  h->amp = nullptr;
  delete h;
  return DQ_OK;
}

int dq_state_num_qubits(dq_state_t h, uint32_t* n) {
  DQ_TRY(check_handle(h));
  if (!n) return fail(DQ_ERR_INVALID_ARG, "null output");
  *n = h->n;
  return DQ_OK;
}

int dq_state_set_basis(dq_state_t h, uint64_t index) {
  DQ_TRY(check_handle_lazy(h));
  if (index >= h->len) return fail(DQ_ERR_INVALID_ARG, "basis index out of range");
  reset_perm(h);
  h->lazy_basis = (int64_t)index;
  return DQ_OK;
}

int dq_state_reset(dq_state_t h) { return dq_state_set_basis(h, 0); }

int dq_state_upload(dq_state_t h, const double* amps, uint64_t len) {
  DQ_TRY(check_handle_lazy(h));
  h->lazy_basis = -1;
  if (!amps || len != h->len) return fail(DQ_ERR_INVALID_ARG, "upload length must be 2^n amplitudes");
  DeviceGuard g(h->device);
  DQ_CUDA_TRY(cudaMemcpyAsync(h->amp, amps, h->bytes, cudaMemcpyHostToDevice, h->stream));
  reset_perm(h);
  return sync_stream(h);
}

int dq_state_download(dq_state_t h, double* amps, uint64_t len) {
  DQ_TRY(check_handle(h));
  if (!amps || len != h->len) return fail(DQ_ERR_INVALID_ARG, "download length must be 2^n amplitudes");
  DeviceGuard g(h->device);
  DQ_TRY(canonicalize(h));
  DQ_CUDA_TRY(cudaMemcpyAsync(amps, h->amp, h->bytes, cudaMemcpyDeviceToHost, h->stream));
  return sync_stream(h);
}

int dq_state_copy(dq_state_t dst, dq_state_t src) {
  DQ_TRY(check_handle_lazy(dst));
  DQ_TRY(check_handle(src));
  dst->lazy_basis = -1;
  if (dst->n != src->n) return fail(DQ_ERR_INVALID_ARG, "state sizes differ");
  DeviceGuard g(dst->device);
  {
    DeviceGuard gs(src->device);
    DQ_TRY(canonicalize(src));
  }
  DQ_TRY(sync_stream(src));
  reset_perm(dst);
  DQ_CUDA_TRY(cudaMemcpyAsync(dst->amp, src->amp, dst->bytes, cudaMemcpyDefault, dst->stream));
  return sync_stream(dst);
}

int dq_state_device_ptr(dq_state_t h, void** dev_ptr, void** stream) {
  DQ_TRY(check_handle(h));
  {
    DeviceGuard g(h->device);
    DQ_TRY(canonicalize(h));
    DQ_TRY(sync_stream(h));
  }
  if (dev_ptr) *dev_ptr = h->amp;
  if (stream) *stream = (void*)h->stream;
  return DQ_OK;
}

int dq_state_synchronize(dq_state_t h) {
  DQ_TRY(check_handle(h));
  DeviceGuard g(h->device);
  return sync_stream(h);
}

int dq_apply_1q(dq_state_t h, const double* u, uint32_t target, uint64_t ctrl_mask,
                uint64_t ctrl_val) {
  DQ_TRY(check_handle(h));
  if (!u) return fail(DQ_ERR_INVALID_ARG, "null matrix");
  if (target >= h->n) return fail(DQ_ERR_INVALID_ARG, "target out of range");
  if (ctrl_mask >> h->n) return fail(DQ_ERR_INVALID_ARG, "control mask outside the register");
  if (ctrl_mask & (1ULL << target)) return fail(DQ_ERR_INVALID_ARG, "control on the target qubit");
  if ((ctrl_val & ~ctrl_mask) != 0) return fail(DQ_ERR_INVALID_ARG, "control value outside the mask");
  if (__builtin_popcountll(ctrl_mask) > 7) return fail(DQ_ERR_INVALID_ARG, "at most 7 controls");
  DeviceGuard g(h->device);
  ctrl_val = map_mask(h, ctrl_val);
  ctrl_mask = map_mask(h, ctrl_mask);
  target = h->perm[target];
  GateOp op;
  op.cls = GC_ONE_Q;
  op.target = target;
  for (int i = 0; i < 4; ++i) op.u[i] = hc{u[2 * i], u[2 * i + 1]};
  if (ctrl_val == ctrl_mask) {
    op.ctrl_mask = ctrl_mask;
    DQ_TRY(launch_gate(h->amp, h->n, op, h->stream, h->device, nullptr));
  } else {
    // controls that must be 0: conjugate by X on those wires (exact permutations)
    const uint64_t zeros = ctrl_mask & ~ctrl_val;
    GateOp x;
    for (uint32_t b = 0; b < h->n; ++b)
      if (zeros >> b & 1ULL) {
        hc xm[4];
        matrix_1q(DQ_X, nullptr, xm);
        classify_1q(xm, b, 0, x);
        DQ_TRY(launch_gate(h->amp, h->n, x, h->stream, h->device, nullptr));
      }
    op.ctrl_mask = ctrl_mask;
    DQ_TRY(launch_gate(h->amp, h->n, op, h->stream, h->device, nullptr));
    for (uint32_t b = 0; b < h->n; ++b)
      if (zeros >> b & 1ULL) {
        hc xm[4];
        matrix_1q(DQ_X, nullptr, xm);
        classify_1q(xm, b, 0, x);
        DQ_TRY(launch_gate(h->amp, h->n, x, h->stream, h->device, nullptr));
      }
  }
  return sync_stream(h);
}

int dq_apply_dense(dq_state_t h, const double* u, const uint32_t* qubits, uint32_t k) {
  DQ_TRY(check_handle(h));
  if (!u || !qubits) return fail(DQ_ERR_INVALID_ARG, "null matrix or qubit list");
  if (k < 1 || k > DQ_MAX_GATE_QUBITS) return fail(DQ_ERR_INVALID_ARG, "k must be in 1..5");
  for (uint32_t a = 0; a < k; ++a) {
    if (qubits[a] >= h->n) return fail(DQ_ERR_INVALID_ARG, "qubit out of range");
    for (uint32_t b = 0; b < a; ++b)
      if (qubits[a] == qubits[b]) return fail(DQ_ERR_INVALID_ARG, "repeated qubit");
  }
  DeviceGuard g(h->device);
  Gate gt;
  gt.k = k;
  const uint32_t dim = 1u << k;
  for (uint32_t i = 0; i < dim * dim; ++i) gt.m[i] = hc{u[2 * i], u[2 * i + 1]};
  for (uint32_t b = 0; b < k; ++b) gt.qubits[b] = h->perm[qubits[b]];
  GateOp op;
  if (k == 1) {
    classify_1q(gt.m, gt.qubits[0], 0, op);
  } else {
    classify(gt, op);
  }
  DQ_TRY(launch_gate(h->amp, h->n, op, h->stream, h->device, nullptr));
  return sync_stream(h);
}

int dq_apply_inst(dq_state_t h, const dq_inst* inst) {
  DQ_TRY(check_handle(h));
  if (!inst) return fail(DQ_ERR_INVALID_ARG, "null instruction");
  DQ_TRY(validate_inst(*inst, h->n, 0, 0, nullptr, 0));
  if (inst->cond_count || inst->kind == DQ_MEASURE || inst->kind == DQ_RESET)
    return fail(DQ_ERR_INVALID_ARG, "dq_apply_inst takes unconditional gates only; use dq_run");
  switch (inst->kind) {
    case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP: return DQ_OK;
    case DQ_G_OPAQUE: case DQ_G_UNSUPPORTED:
      return fail(DQ_ERR_UNSUPPORTED, "unsupported generic gate");
    default: break;
  }
  DeviceGuard g(h->device);
  dq_inst mapped = *inst;
  for (int i = 0; i < mapped.nq && i < DQ_MAX_INST_QUBITS; ++i)
    if (mapped.q[i] >= 0 && (uint32_t)mapped.q[i] < h->n) mapped.q[i] = (int32_t)h->perm[mapped.q[i]];
  GateOp op;
  if (!inst_to_op(mapped, op)) return fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
  DQ_TRY(launch_gate(h->amp, h->n, op, h->stream, h->device, nullptr));
  return sync_stream(h);
}

int dq_measure_p1(dq_state_t h, uint32_t qubit, double* p1) {
  DQ_TRY(check_handle(h));
  if (!p1 || qubit >= h->n) return fail(DQ_ERR_INVALID_ARG, "bad qubit or null output");
  DeviceGuard g(h->device);
  double* d = h->sc.d_partial + kPartials - 1;
  DQ_TRY(launch_p1(h->amp, h->n, h->perm[qubit], h->sc, d, h->stream, h->device));
  return read_scalars(h, d, 1, p1);
}

int dq_collapse(dq_state_t h, uint32_t qubit, int outcome, double p1) {
  DQ_TRY(check_handle(h));
  if (qubit >= h->n || (outcome != 0 && outcome != 1))
    return fail(DQ_ERR_INVALID_ARG, "bad qubit or outcome");
  DeviceGuard g(h->device);
  double norm;
  if (outcome == 1) {
    norm = sqrt(p1);
    if (norm < 1e-15) norm = 1e-15;
  } else {
    double t = 1.0 - p1;
    if (t < 0.0) t = 0.0;
    norm = sqrt(t);
    if (norm < 1e-15) norm = 1e-15;
  }
  DQ_TRY(launch_collapse(h->amp, h->n, h->perm[qubit], outcome, norm, h->stream, h->device));
  return sync_stream(h);
}

int dq_measure(dq_state_t h, uint32_t qubit, double r, int* outcome, double* p1_out) {
  double p1 = 0.0;
  DQ_TRY(dq_measure_p1(h, qubit, &p1));
  const int o = (r < p1) ? 1 : 0;
  DQ_TRY(dq_collapse(h, qubit, o, p1));
  if (outcome) *outcome = o;
  if (p1_out) *p1_out = p1;
  return DQ_OK;
}

int dq_run(dq_state_t h, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
           uint64_t nconds, uint64_t seed, int32_t* cbits, uint64_t ncbits,
           const dq_run_opts* opts, dq_profile* prof) {
  DQ_TRY(check_handle_lazy(h));
  if (ninst && !prog) return fail(DQ_ERR_INVALID_ARG, "null program");
  if (ncbits && !cbits) return fail(DQ_ERR_INVALID_ARG, "null cbits");
  dq_run_opts o{};
  if (opts) o = *opts;
  if (o.semantics != DQ_SEM_SIMULATE && o.semantics != DQ_SEM_SHOTS)
    return fail(DQ_ERR_INVALID_ARG, "unknown semantics");
  if (o.exec != DQ_EXEC_PER_GATE && o.exec != DQ_EXEC_FUSED)
    return fail(DQ_ERR_INVALID_ARG, "unknown exec mode");
  for (uint64_t i = 0; i < ninst; ++i)
    DQ_TRY(validate_inst(prog[i], h->n, nconds, ncbits, conds, i));
  DeviceGuard g(h->device);
  const auto t0 = std::chrono::steady_clock::now();
  RunCtx c;
  c.h = h;
  c.rng.seed(seed);
  c.cbits = cbits;
  c.ncbits = ncbits;
  memset(&c.prof, 0, sizeof(c.prof));
  c.prof.failed_inst = -1;
  c.sem = o.semantics;
  c.timer.on = o.profile != 0;
  c.timer.st = h->stream;
  int rc = DQ_OK;
  const bool fused = o.exec == DQ_EXEC_FUSED && !o.profile && h->n >= kFusedMinQubits;
  if (fused) {
    FusedHooks hooks;
    hooks.measure = [&c, h](uint32_t q, int* out) {
      DQ_TRY(materialize_basis(h));
      return do_measure(c, q, out);
    };
    hooks.exact_gate = [&c, h](const GateOp& op) {
      DQ_TRY(materialize_basis(h));
      return do_gate_op(c, op, 0);
    };
    hooks.lazy_basis = &h->lazy_basis;
    hooks.cbits = cbits;
    hooks.ncbits = ncbits;
    hooks.conds = conds;
    rc = fused_run(h->amp, h->n, prog, ninst, o, h->fw, h->stream, h->device, hooks, &c.prof,
                   h->perm);
    update_permuted(h);
  } else if ((rc = canonicalize(h)) != DQ_OK) {
    // error already recorded
  } else if (o.semantics == DQ_SEM_SHOTS) {
    const std::vector<FusedEntry> fused = fuse_program(prog, ninst, h->n);
    for (const FusedEntry& e : fused) {
      if (e.inst < 0) {
        GateOp op;
        classify_1q(e.m, e.qubit, 0, op);
        rc = do_gate_op(c, op, 0);
      } else {
        const dq_inst& in = prog[e.inst];
        if (!cond_holds(in, conds, cbits, ncbits)) continue;
        rc = exec_inst(c, in);
      }
      if (rc != DQ_OK) {
        c.prof.failed_inst = e.inst;
        break;
      }
    }
  } else {
    for (uint64_t i = 0; i < ninst; ++i) {
      const dq_inst& in = prog[i];
      if (!cond_holds(in, conds, cbits, ncbits)) continue;
      rc = exec_inst(c, in);
      if (rc != DQ_OK) {
        c.prof.failed_inst = (int64_t)i;
        break;
      }
    }
  }
  if (rc == DQ_OK) rc = sync_stream(h);
  const auto t1 = std::chrono::steady_clock::now();
  c.prof.total_time = std::chrono::duration<double>(t1 - t0).count();
  c.timer.collect(&c.prof);
  if (prof) *prof = c.prof;
  return rc;
}

int dq_marginal_probs(dq_state_t h, const uint32_t* qubits, uint32_t k, double* out) {
  DQ_TRY(check_handle(h));
  if (!out || (k && !qubits)) return fail(DQ_ERR_INVALID_ARG, "null argument");
  if (k > h->n || k > 30) return fail(DQ_ERR_INVALID_ARG, "too many marginal qubits");
  for (uint32_t a = 0; a < k; ++a) {
    if (qubits[a] >= h->n) return fail(DQ_ERR_INVALID_ARG, "qubit out of range");
    for (uint32_t b = 0; b < a; ++b)
      if (qubits[a] == qubits[b]) return fail(DQ_ERR_INVALID_ARG, "repeated qubit");
  }
  DeviceGuard g(h->device);
  std::vector<uint32_t> mq(qubits, qubits + k);
  for (auto& q : mq) q = h->perm[q];
  qubits = mq.data();
  const uint64_t nj = 1ULL << k;
  // small outputs land in the handle's pinned buffer (then one memcpy), large
  // ones go straight to the caller's memory
  const bool staged = nj <= (1ULL << 16);
  // output first, the reduction's partials 256-byte aligned after it
  const size_t out_bytes = (sizeof(double) * nj + 255) / 256 * 256;
  const size_t work_bytes = sizeof(double) * marginal_workspace(h->n, qubits, k, h->device);
  QueryBuffer qb;
  DQ_TRY(qb.get(h, out_bytes + work_bytes));
  if (staged) DQ_TRY(ensure_query_buffers(h, 0, sizeof(double) * nj));
  double* d = reinterpret_cast<double*>(qb.ptr);
  double* work = work_bytes ? reinterpret_cast<double*>(reinterpret_cast<char*>(qb.ptr) + out_bytes)
                            : nullptr;
  DQ_TRY(launch_marginal(h->amp, h->n, qubits, k, d, work, h->sc, h->stream, h->device));
  DQ_CUDA_TRY(cudaMemcpyAsync(staged ? h->q_host : (void*)out, d, sizeof(double) * nj,
                              cudaMemcpyDeviceToHost, h->stream));
  DQ_TRY(sync_stream(h));
  if (staged) memcpy(out, h->q_host, sizeof(double) * nj);
  return DQ_OK;
}

int dq_sample_key(dq_state_t h, const uint32_t* qubits, uint32_t k, const uint32_t* key8,
                  uint64_t shots, uint32_t* out_idx, uint64_t* n_boundary) {
  DQ_TRY(check_handle(h));
  if (!key8 || (shots && !out_idx) || (k && !qubits))
    return fail(DQ_ERR_INVALID_ARG, "null argument");
  if (k > h->n || k > 30) return fail(DQ_ERR_INVALID_ARG, "too many sampled qubits");
  for (uint32_t a = 0; a < k; ++a) {
    if (qubits[a] >= h->n) return fail(DQ_ERR_INVALID_ARG, "qubit out of range");
    for (uint32_t b = 0; b < a; ++b)
      if (qubits[a] == qubits[b]) return fail(DQ_ERR_INVALID_ARG, "repeated qubit");
  }
  DeviceGuard g(h->device);
  std::vector<uint32_t> mq(qubits, qubits + k);
  for (auto& q : mq) q = h->perm[q];
  qubits = mq.data();
  const uint64_t nj = 1ULL << k;
  // CDF, sampled indices and the reductions' workspace in the handle's device
  // query buffer, each part 256-byte aligned
  auto align256 = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t cdf_bytes = align256(sizeof(double) * nj);
  const size_t idx_bytes = align256(sizeof(uint32_t) * (shots ? shots : 1));
  const size_t work_bytes = sizeof(double) * std::max<uint64_t>(marginal_workspace(h->n, qubits, k, h->device),
                                                                cdf_workspace(nj));
  QueryBuffer qb;
  DQ_TRY(qb.get(h, cdf_bytes + idx_bytes + work_bytes));
  char* base = reinterpret_cast<char*>(qb.ptr);
  double* cdf = reinterpret_cast<double*>(base);
  uint32_t* idx = reinterpret_cast<uint32_t*>(base + cdf_bytes);
  double* work = reinterpret_cast<double*>(base + cdf_bytes + idx_bytes);
  int rc = launch_marginal(h->amp, h->n, qubits, k, cdf, work, h->sc, h->stream, h->device);
  cudaError_t e = cudaSuccess;
  if (rc == DQ_OK) rc = launch_cdf(cdf, nj, work, h->stream, h->device);
  if (rc == DQ_OK) {
    e = cudaMemsetAsync(h->sc.d_ull, 0, sizeof(unsigned long long), h->stream);
    if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
  }
  if (rc == DQ_OK) rc = launch_sample(cdf, nj, key8, shots, idx, h->sc.d_ull, h->stream, h->device);
  if (rc == DQ_OK && shots) {
    e = cudaMemcpyAsync(out_idx, idx, sizeof(uint32_t) * shots, cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
  }
  unsigned long long nb = 0;
  if (rc == DQ_OK) {
    e = cudaMemcpyAsync(h->sc.h_pinned, h->sc.d_ull, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
  }
  if (rc != DQ_OK) return rc;
  DQ_TRY(sync_stream(h));
  memcpy(&nb, h->sc.h_pinned, sizeof(nb));
  if (n_boundary) *n_boundary = nb;
  return DQ_OK;
}

int dq_sample(dq_state_t h, const uint32_t* qubits, uint32_t k, uint64_t seed, uint64_t shots,
              uint32_t* out_idx, uint64_t* n_boundary) {
  uint32_t key[8];
  seed_key_from_u64(seed, key);
  return dq_sample_key(h, qubits, k, key, shots, out_idx, n_boundary);
}

int dq_inner(dq_state_t h, const double* other, uint64_t len, double* re, double* im) {
  DQ_TRY(check_handle(h));
  if (!other || !re || !im) return fail(DQ_ERR_INVALID_ARG, "null argument");
  if (len != h->len) return fail(DQ_ERR_INVALID_ARG, "length mismatch");
  DeviceGuard g(h->device);
  DQ_TRY(canonicalize(h));
  double2* d = nullptr;
  DQ_CUDA_TRY(pool_malloc_async((void**)&d, h->bytes, h->stream));
  int rc = DQ_OK;
  cudaError_t e = cudaMemcpyAsync(d, other, h->bytes, cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
  double* dout = h->sc.d_partial + kPartials - 2;
  if (rc == DQ_OK) rc = launch_inner(h->amp, d, h->n, h->sc, dout, h->stream, h->device);
  double v[2] = {0, 0};
  if (rc == DQ_OK) rc = read_scalars(h, dout, 2, v);
  cudaFreeAsync(d, h->stream);
  DQ_TRY(rc);
  DQ_TRY(sync_stream(h));
  *re = v[0];
  *im = v[1];
  return DQ_OK;
}

int dq_norm_sqr(dq_state_t h, double* out) {
  DQ_TRY(check_handle(h));
  if (!out) return fail(DQ_ERR_INVALID_ARG, "null output");
  DeviceGuard g(h->device);
  double* d = h->sc.d_partial + kPartials - 1;
  DQ_TRY(launch_norm(h->amp, h->n, h->sc, d, h->stream, h->device));
  return read_scalars(h, d, 1, out);
}

int dq_debug_plan(uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_run_opts* opts,
                  uint8_t* out, uint64_t cap, uint64_t* len) {
  if (!len || (ninst && !prog)) return fail(DQ_ERR_INVALID_ARG, "null argument");
  if (n < kFusedMinQubits || n > kMaxQubits)
    return fail(DQ_ERR_INVALID_ARG, "fused planning needs 10..34 qubits");
  dq_run_opts o{};
  if (opts) o = *opts;
  o.exec = DQ_EXEC_FUSED;
  for (uint64_t i = 0; i < ninst; ++i) {
    DQ_TRY(validate_inst(prog[i], n, 0, 0, nullptr, i));
    if (prog[i].cond_count) return fail(DQ_ERR_INVALID_ARG, "plan-only mode takes unitary programs");
  }
  FusedWork fw;
  std::vector<uint8_t> blob;
  std::vector<uint64_t> offs;
  fw.plan_out = &blob;
  fw.plan_offs = &offs;
  FusedHooks hooks;
  dq_profile prof{};
  uint32_t perm[64];
  for (uint32_t l = 0; l < 64; ++l) perm[l] = l;
  DQ_TRY(fused_run(nullptr, n, prog, ninst, o, fw, nullptr, 0, hooks, &prof, perm));
  const uint64_t hdr = 16 + 4 * 64 + 8 * offs.size();
  const uint64_t need = hdr + blob.size();
  *len = need;
  if (!out || cap < need) return out ? fail(DQ_ERR_INVALID_ARG, "output buffer too small") : DQ_OK;
  uint32_t h4[4] = {0x4C505144u, (uint32_t)offs.size(), fw.plan_rb, 0};
  memcpy(out, h4, 16);
  memcpy(out + 16, perm, 4 * 64);
  memcpy(out + 16 + 256, offs.data(), 8 * offs.size());
  memcpy(out + hdr, blob.data(), blob.size());
  return DQ_OK;
}

int dq_rng_f64(uint64_t seed, uint64_t skip, uint64_t count, double* out) {
  if (count && !out) return fail(DQ_ERR_INVALID_ARG, "null output");
  uint32_t key[8];
  seed_key_from_u64(seed, key);
  for (uint64_t i = 0; i < count; ++i) out[i] = chacha8_draw(key, skip + i);
  return DQ_OK;
}

int dq_rng_seed_key(uint64_t seed, uint32_t* key8) {
  if (!key8) return fail(DQ_ERR_INVALID_ARG, "null output");
  seed_key_from_u64(seed, key8);
  return DQ_OK;
}

int dq_chacha_block(const uint32_t* in16, uint32_t rounds, uint32_t* out16) {
  if (!in16 || !out16 || rounds == 0 || (rounds & 1)) return fail(DQ_ERR_INVALID_ARG, "bad arguments");
  chacha_block(in16, rounds, out16);
  return DQ_OK;
}

}  // extern "C"
