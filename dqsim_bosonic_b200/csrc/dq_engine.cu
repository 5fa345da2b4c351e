// dq_engine.cu — exact per-gate kernels, measurement reductions, marginal
// probabilities, the device CDF and the per-shot sampler.
//
// Per-gate kernels restate src/engine.rs (apply_one_qubit 24-101,
// apply_n_qubit 109-181) with the num-complex operation order and no FMA, so
// each gate's output equals the Rust engine's bit for bit.  Instead of the
// reference's filter over all 2^n indices, every kernel enumerates only the
// amplitudes the gate changes (zero bits inserted at the target/control
// positions), so a gate with c controls moves 2^-c of the state.
#include <cuda_runtime.h>

#include <algorithm>

#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_reduce.cuh"
#include "dq_rng.cuh"

namespace dq {

namespace {

constexpr int kThreads = 256;

struct Pos {
  uint32_t p[8];
  int np;
};

// Callers guarantee popcount(mask) <= 8 (gates touch at most 5 qubits;
// dq_apply_1q limits its controls); extra bits are never written past p[7].
Pos make_pos(uint64_t mask) {
  Pos ps{};
  ps.np = 0;
  for (uint32_t b = 0; b < 64 && ps.np < 8; ++b)
    if (mask >> b & 1ULL) ps.p[ps.np++] = b;
  return ps;
}

inline unsigned blocks_for(uint64_t items, unsigned threads) {
  uint64_t b = (items + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 0x7fffffffULL) b = 0x7fffffffULL;
  return (unsigned)b;
}

// ---- one-qubit family --------------------------------------------------------

__global__ void k_one_q(double2* __restrict__ s, uint64_t count, Pos pos, uint64_t setb,
                        uint64_t tbit, double2 u00, double2 u01, double2 u10, double2 u11) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint64_t i = insert_zeros(k, pos.p, pos.np) | setb;
  const uint64_t j = i | tbit;
  const double2 a = s[i], b = s[j];
  s[i] = cadd_x(cmul_x(u00, a), cmul_x(u01, b));
  s[j] = cadd_x(cmul_x(u10, a), cmul_x(u11, b));
}

__global__ void k_phase(double2* __restrict__ s, uint64_t count, Pos pos, uint64_t setb,
                        double2 e) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint64_t i = insert_zeros(k, pos.p, pos.np) | setb;
  s[i] = cmul_x(e, s[i]);
}

__global__ void k_exchange(double2* __restrict__ s, uint64_t count, Pos pos, uint64_t seta,
                           uint64_t setb) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint64_t base = insert_zeros(k, pos.p, pos.np);
  const uint64_t i = base | seta, j = base | setb;
  const double2 a = s[i], b = s[j];
  s[i] = b;
  s[j] = a;
}

// ---- k-qubit diagonal and dense -----------------------------------------------

struct DiagParams {
  double2 d[32];
  uint32_t q[5];   // q[0] = MSB of the diagonal index
  uint32_t k;
};

__global__ void k_diag(double2* __restrict__ s, uint64_t count, DiagParams P) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t g = 0;
  for (uint32_t b = 0; b < P.k; ++b) g = (g << 1) | (uint32_t)((i >> P.q[b]) & 1ULL);
  const double2 d = P.d[g];
  if (d.x == 1.0 && d.y == 0.0) return;   // 1 * v == v exactly
  s[i] = cmul_x(d, s[i]);
}

template <int K>
struct DenseParams {
  double2 m[(1 << K) * (1 << K)];
  uint64_t off[1 << K];
  Pos pos;
};

template <int K>
__global__ void k_dense(double2* __restrict__ s, uint64_t count, DenseParams<K> P) {
  constexpr int D = 1 << K;
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint64_t base = insert_zeros(k, P.pos.p, P.pos.np);
  double2 v[D];
#pragma unroll
  for (int j = 0; j < D; ++j) v[j] = s[base + P.off[j]];
#pragma unroll 1
  for (int r = 0; r < D; ++r) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const double2 u = P.m[r * D + c];
      if (u.x != 0.0 || u.y != 0.0) acc = cadd_x(acc, cmul_x(u, v[c]));
    }
    s[base + P.off[r]] = acc;
  }
}

template <int K>
int launch_dense_k(double2* s, uint32_t n, const Gate& g, cudaStream_t st) {
  DenseParams<K> P;
  constexpr int D = 1 << K;
  uint64_t mask = 0;
  for (int b = 0; b < K; ++b) mask |= 1ULL << g.qubits[b];
  for (int j = 0; j < D; ++j) {
    uint64_t off = 0;
    for (int b = 0; b < K; ++b)
      if ((j >> (K - 1 - b)) & 1) off |= 1ULL << g.qubits[b];
    P.off[j] = off;
  }
  for (int i = 0; i < D * D; ++i) P.m[i] = make_double2(g.m[i].re, g.m[i].im);
  P.pos = make_pos(mask);
  const uint64_t count = 1ULL << (n - K);
  k_dense<K><<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, P);
  return DQ_OK;
}

__global__ void k_p1(const double2* __restrict__ s, uint64_t count, uint32_t q,
                     double* partial, unsigned* counter, double* out) {
  double acc = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t bit = 1ULL << q;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += stride)
    acc = __dadd_rn(acc, norm_sqr_x(s[insert_zero(k, q) | bit]));
  double v[1] = {acc};
  finish_partials<1>(v, partial, counter, out);
}

__global__ void k_norm(const double2* __restrict__ s, uint64_t count, double* partial,
                       unsigned* counter, double* out) {
  double acc = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += stride)
    acc = __dadd_rn(acc, norm_sqr_x(s[i]));
  double v[1] = {acc};
  finish_partials<1>(v, partial, counter, out);
}

// sum conj(a_i) * b_i  (SimulationResult::fidelity, simulator.rs:184-191)
__global__ void k_inner(const double2* __restrict__ a, const double2* __restrict__ b,
                        uint64_t count, double* partial, unsigned* counter, double* out) {
  double re = 0.0, im = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += stride) {
    const double2 x = a[i], y = b[i];
    const double2 p = cmul_x(make_double2(x.x, -x.y), y);
    re = __dadd_rn(re, p.x);
    im = __dadd_rn(im, p.y);
  }
  double v[2] = {re, im};
  finish_partials<2>(v, partial, counter, out);
}

unsigned red_blocks(uint64_t items, int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint64_t want = (items + kRedThreads - 1) / kRedThreads;
  // W * grid partials stay below kPartials - 8, clear of the result slots
  uint64_t cap = (uint64_t)sms * 4;
  if (cap > (uint64_t)kPartials / 4) cap = kPartials / 4;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (unsigned)want;
}

// ---- collapse / init ------------------------------------------------------------------

__global__ void k_collapse(double2* __restrict__ s, uint64_t count, uint64_t bit, int outcome,
                           double norm) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const bool set = (i & bit) != 0;
  if (set != (outcome == 1)) {
    s[i] = make_double2(0.0, 0.0);
  } else {
    const double2 a = s[i];
    s[i] = make_double2(__ddiv_rn(a.x, norm), __ddiv_rn(a.y, norm));
  }
}

__global__ void k_set_basis(double2* __restrict__ s, uint64_t count, uint64_t index) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  s[i] = make_double2(i == index ? 1.0 : 0.0, 0.0);
}

// ---- marginal probabilities -----------------------------------------------------------
//
// marginal_probs (engine.rs:368-390): out[j] = sum of |psi_i|^2 over i whose
// marginal bits spell j (qubits[0] = MSB of j), in ascending i.  When each
// output has few terms a thread owns one j and adds its terms in ascending
// i, which is exactly the reference's sum.  Otherwise (S, j) segments are
// reduced by blocks and the segment partials summed in order.

struct Pos32 {
  uint32_t p[32];
  int np;
};

struct MargParams {
  uint32_t q[32];     // marginal qubits, q[0] = MSB of j
  Pos32 rest;         // the marginal qubits, ascending (zero bits inserted there)
  uint32_t k;
};

__device__ __forceinline__ uint64_t deposit_j(uint64_t j, const MargParams& P) {
  uint64_t bits = 0;
  for (uint32_t b = 0; b < P.k; ++b) bits |= ((j >> (P.k - 1 - b)) & 1ULL) << P.q[b];
  return bits;
}

__global__ void k_marg_thread(const double2* __restrict__ s, uint64_t nj, uint64_t nterms,
                              MargParams P, double* __restrict__ out) {
  const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= nj) return;
  const uint64_t jb = deposit_j(j, P);
  double acc = 0.0;
  for (uint64_t r = 0; r < nterms; ++r)
    acc = __dadd_rn(acc, norm_sqr_x(s[insert_zeros(r, P.rest.p, P.rest.np) | jb]));
  out[j] = acc;
}

// One block sums segment `seg` of output j.  When the lowest marginal qubit
// c leaves runs of at least a block of consecutive amplitudes (indices whose
// bits above c agree), a run's base index is computed once and the run is
// streamed.  Otherwise (marginal qubits at low positions, e.g. after a
// relabeling) every thread takes terms r = r0 + tid, + blockDim, ... and
// finds the index from shared tables that deposit 7 bits of r at a time.
// Four independent partial sums per thread, combined in a fixed order, then a
// fixed-order block sum: deterministic.
__global__ void k_marg_seg(const double2* __restrict__ s, uint64_t nterms, uint32_t nseg,
                           MargParams P, double* __restrict__ partial) {
  __shared__ uint64_t tab[5][128];
  const uint64_t j = blockIdx.x / nseg;
  const uint32_t seg = blockIdx.x % nseg;
  const uint64_t per = nterms / nseg;  // nseg is a power of two dividing nterms
  const uint64_t r0 = (uint64_t)seg * per;
  const uint64_t jb = deposit_j(j, P);
  const uint32_t c = P.rest.np ? P.rest.p[0] : 63u;
  const uint64_t run = c >= 63u ? per : (per < (1ULL << c) ? per : (1ULL << c));
  const uint32_t bd = blockDim.x;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  if (run >= bd) {
    for (uint64_t rb = r0; rb < r0 + per; rb += run) {
      const double2* src = s + (insert_zeros(rb, P.rest.p, P.rest.np) | jb);
      uint64_t off = threadIdx.x;
      for (; off + 3ULL * bd < run; off += 4ULL * bd) {
        a0 = __dadd_rn(a0, norm_sqr_x(src[off]));
        a1 = __dadd_rn(a1, norm_sqr_x(src[off + bd]));
        a2 = __dadd_rn(a2, norm_sqr_x(src[off + 2ULL * bd]));
        a3 = __dadd_rn(a3, norm_sqr_x(src[off + 3ULL * bd]));
      }
      for (; off < run; off += bd) a0 = __dadd_rn(a0, norm_sqr_x(src[off]));
    }
  } else {
    // deposit tables: tab[g][v] = index bits of the term v << 7g
    uint32_t bits = 0;
    while (bits < 64 && (1ULL << bits) < nterms) ++bits;
    const uint32_t ntab = min((bits + 6) / 7, 5u);  // nterms <= 2^34 needs at most 5
    for (uint32_t i = threadIdx.x; i < ntab * 128u; i += bd)
      tab[i >> 7][i & 127u] = insert_zeros((uint64_t)(i & 127u) << (7u * (i >> 7)), P.rest.p,
                                           P.rest.np);
    __syncthreads();
    auto index = [&](uint64_t r) {
      uint64_t x = jb;
      for (uint32_t g = 0; g < ntab; ++g) x |= tab[g][(r >> (7u * g)) & 127u];
      return x;
    };
    uint64_t e = threadIdx.x;
    for (; e + 3ULL * bd < per; e += 4ULL * bd) {
      const uint64_t r = r0 + e;
      a0 = __dadd_rn(a0, norm_sqr_x(s[index(r)]));
      a1 = __dadd_rn(a1, norm_sqr_x(s[index(r + bd)]));
      a2 = __dadd_rn(a2, norm_sqr_x(s[index(r + 2ULL * bd)]));
      a3 = __dadd_rn(a3, norm_sqr_x(s[index(r + 3ULL * bd)]));
    }
    for (; e < per; e += bd) a0 = __dadd_rn(a0, norm_sqr_x(s[index(r0 + e)]));
  }
  double acc = __dadd_rn(__dadd_rn(a0, a1), __dadd_rn(a2, a3));
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Marginal qubits all among the low 10 bits: block b streams the contiguous
// chunk [b * chunk, (b + 1) * chunk) fully coalesced, thread t summing the
// elements whose low 10 bits equal t; output j then adds, in ascending t, the
// threads whose bits at the marginal positions spell j.  partial[j * gridDim.x + b].
__global__ void __launch_bounds__(1024) k_marg_low(const double2* __restrict__ s, uint64_t chunk,
                                                   MargParams P, double* __restrict__ partial) {
  __shared__ double sh[1024];
  const uint32_t t = threadIdx.x;
  const double2* src = s + (uint64_t)blockIdx.x * chunk + t;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  uint64_t i = 0;
  for (; i + 3 * 1024 < chunk; i += 4 * 1024) {
    a0 = __dadd_rn(a0, norm_sqr_x(src[i]));
    a1 = __dadd_rn(a1, norm_sqr_x(src[i + 1024]));
    a2 = __dadd_rn(a2, norm_sqr_x(src[i + 2048]));
    a3 = __dadd_rn(a3, norm_sqr_x(src[i + 3072]));
  }
  for (; i < chunk; i += 1024) a0 = __dadd_rn(a0, norm_sqr_x(src[i]));
  sh[t] = __dadd_rn(__dadd_rn(a0, a1), __dadd_rn(a2, a3));
  __syncthreads();
  const uint64_t nj = 1ULL << P.k;
  if (t < nj) {
    const uint32_t jb = (uint32_t)deposit_j(t, P);
    const uint32_t nr = 1024u >> P.k;
    double acc = 0.0;
    for (uint32_t r = 0; r < nr; ++r)
      acc = __dadd_rn(acc, sh[(uint32_t)insert_zeros(r, P.rest.p, P.rest.np) | jb]);
    partial[(uint64_t)t * gridDim.x + blockIdx.x] = acc;
  }
}

__global__ void k_marg_sum(const double* __restrict__ partial, uint64_t nj, uint32_t nseg,
                           double* __restrict__ out) {
  const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= nj) return;
  double acc = 0.0;
  for (uint32_t g = 0; g < nseg; ++g) acc = __dadd_rn(acc, partial[j * nseg + g]);
  out[j] = acc;
}

// ---- CDF (inclusive prefix sum) and sampling ----------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;                       // elements per thread
constexpr int kScanChunk = kScanThreads * kScanPer;

// Exclusive scan of per-thread values across the block (fixed order).
__device__ double block_exclusive_scan(double v, double* total) {
  __shared__ double sh[kScanThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc = __dadd_rn(inc, t);
  }
  __syncthreads();
  if (lane == 31) sh[w] = inc;
  __syncthreads();
  double woff = 0.0, tot = 0.0;
  for (int i = 0; i < kScanThreads / 32; ++i) {
    if (i < w) woff = __dadd_rn(woff, sh[i]);
    tot = __dadd_rn(tot, sh[i]);
  }
  *total = tot;
  double exw = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exw = 0.0;
  (void)v;
  return __dadd_rn(woff, exw);
}

__device__ __forceinline__ double thread_segment_sum(const double* d, uint64_t len, uint64_t b0) {
  double a = 0.0;
#pragma unroll
  for (int e = 0; e < kScanPer; ++e) {
    const uint64_t i = b0 + e;
    if (i < len) a = __dadd_rn(a, d[i]);
  }
  return a;
}

__global__ void k_scan_sums(const double* __restrict__ d, uint64_t len, double* __restrict__ sums) {
  const uint64_t b0 = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanPer;
  double tot;
  (void)block_exclusive_scan(thread_segment_sum(d, len, b0), &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single block: in-place exclusive scan of sums[nb], looping with a carry.
__global__ void k_scan_offsets(double* __restrict__ sums, uint64_t nb) {
  __shared__ double carry;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  for (uint64_t base = 0; base < nb; base += kScanThreads) {
    const uint64_t i = base + threadIdx.x;
    const double v = i < nb ? sums[i] : 0.0;
    double tot;
    const double ex = block_exclusive_scan(v, &tot);
    const double c = carry;
    if (i < nb) sums[i] = __dadd_rn(c, ex);
    __syncthreads();
    if (threadIdx.x == 0) carry = __dadd_rn(c, tot);
    __syncthreads();
  }
}

__global__ void k_scan_apply(double* __restrict__ d, uint64_t len, const double* __restrict__ offs) {
  const uint64_t b0 = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanPer;
  double tot;
  const double ex = block_exclusive_scan(thread_segment_sum(d, len, b0), &tot);
  double run = __dadd_rn(offs[blockIdx.x], ex);
#pragma unroll
  for (int e = 0; e < kScanPer; ++e) {
    const uint64_t i = b0 + e;
    if (i < len) {
      run = __dadd_rn(run, d[i]);
      d[i] = run;
    }
  }
}

__global__ void k_set_last_one(double* d, uint64_t len) { d[len - 1] = 1.0; }

struct Key8 {
  uint32_t k[8];
};

// sample_counts inner loop (engine.rs:426-431) with draw s computed from the
// stream position: idx = partition_point(cdf < r).min(len - 1).
__global__ void k_sample(const double* __restrict__ cdf, uint64_t len, Key8 key, uint64_t shots,
                         uint32_t* __restrict__ out, unsigned long long* __restrict__ nboundary) {
  const uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (s >= shots) return;
  const double r = chacha8_draw(key.k, s);
  uint64_t lo = 0, hi = len;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (cdf[mid] < r) lo = mid + 1; else hi = mid;
  }
  if (lo > len - 1) lo = len - 1;
  out[s] = (uint32_t)lo;
  const double up = cdf[lo];
  bool near = fabs(up - r) <= 1e-12;
  if (lo > 0) near = near || fabs(r - cdf[lo - 1]) <= 1e-12;
  if (near) atomicAdd(nboundary, 1ULL);
}

}  // namespace

unsigned grid_for(uint64_t work, unsigned threads, int device) {
  (void)device;
  return blocks_for(work, threads);
}

int launch_gate(double2* s, uint32_t n, const GateOp& op, cudaStream_t st, int device,
                uint64_t* launches) {
  (void)device;
  auto d2 = [](hc z) { return make_double2(z.re, z.im); };
  switch (op.cls) {
    case GC_ONE_Q: {
      const uint64_t tb = 1ULL << op.target;
      const Pos pos = make_pos(op.ctrl_mask | tb);
      const uint64_t count = 1ULL << (n - pos.np);
      k_one_q<<<blocks_for(count, kThreads), kThreads, 0, st>>>(
          s, count, pos, op.ctrl_mask, tb, d2(op.u[0]), d2(op.u[1]), d2(op.u[2]), d2(op.u[3]));
      break;
    }
    case GC_PHASE: {
      const uint64_t tb = 1ULL << op.target;
      const Pos pos = make_pos(op.ctrl_mask | tb);
      const uint64_t count = 1ULL << (n - pos.np);
      k_phase<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, pos, op.ctrl_mask | tb,
                                                                 d2(op.u[0]));
      break;
    }
    case GC_XPERM: {
      const uint64_t tb = 1ULL << op.target;
      const Pos pos = make_pos(op.ctrl_mask | tb);
      const uint64_t count = 1ULL << (n - pos.np);
      k_exchange<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, pos, op.ctrl_mask,
                                                                    op.ctrl_mask | tb);
      break;
    }
    case GC_SWAP: {
      const uint64_t ta = 1ULL << op.target, tb = 1ULL << op.target2;
      const Pos pos = make_pos(op.ctrl_mask | ta | tb);
      const uint64_t count = 1ULL << (n - pos.np);
      k_exchange<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, pos,
                                                                    op.ctrl_mask | tb,
                                                                    op.ctrl_mask | ta);
      break;
    }
    case GC_DIAG: {
      DiagParams P{};
      const Gate& g = op.dense;
      const uint32_t dim = 1u << g.k;
      for (uint32_t i = 0; i < dim; ++i) P.d[i] = d2(g.m[i * dim + i]);
      for (uint32_t b = 0; b < g.k; ++b) P.q[b] = g.qubits[b];
      P.k = g.k;
      const uint64_t count = 1ULL << n;
      k_diag<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, P);
      break;
    }
    case GC_DENSE: {
      const Gate& g = op.dense;
      switch (g.k) {
        case 1: DQ_TRY(launch_dense_k<1>(s, n, g, st)); break;
        case 2: DQ_TRY(launch_dense_k<2>(s, n, g, st)); break;
        case 3: DQ_TRY(launch_dense_k<3>(s, n, g, st)); break;
        case 4: DQ_TRY(launch_dense_k<4>(s, n, g, st)); break;
        case 5: DQ_TRY(launch_dense_k<5>(s, n, g, st)); break;
        default: return fail(DQ_ERR_INTERNAL, "dense gate with k outside 1..5");
      }
      break;
    }
    default:
      return fail(DQ_ERR_INTERNAL, "unclassified gate");
  }
  if (launches) ++*launches;
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

unsigned p1_reduction_blocks(uint32_t n, int device) { return red_blocks(1ULL << (n - 1), device); }
unsigned reduction_blocks(uint64_t items, int device) { return red_blocks(items, device); }

int launch_p1(const double2* s, uint32_t n, uint32_t q, Scratch& sc, double* d_out,
              cudaStream_t st, int device) {
  const uint64_t count = 1ULL << (n - 1);
  k_p1<<<red_blocks(count, device), kRedThreads, 0, st>>>(s, count, q, sc.d_partial,
                                                          sc.d_counter, d_out);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int launch_norm(const double2* a, uint32_t n, Scratch& sc, double* d_out, cudaStream_t st,
                int device) {
  const uint64_t count = 1ULL << n;
  k_norm<<<red_blocks(count, device), kRedThreads, 0, st>>>(a, count, sc.d_partial, sc.d_counter,
                                                            d_out);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int launch_inner(const double2* a, const double2* b, uint32_t n, Scratch& sc, double* d_out,
                 cudaStream_t st, int device) {
  const uint64_t count = 1ULL << n;
  k_inner<<<red_blocks(count, device), kRedThreads, 0, st>>>(a, b, count, sc.d_partial,
                                                             sc.d_counter, d_out);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int launch_collapse(double2* s, uint32_t n, uint32_t q, int outcome, double norm,
                    cudaStream_t st, int device) {
  (void)device;
  const uint64_t count = 1ULL << n;
  k_collapse<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, 1ULL << q, outcome, norm);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int launch_set_basis(double2* s, uint32_t n, uint64_t index, cudaStream_t st, int device) {
  (void)device;
  const uint64_t count = 1ULL << n;
  k_set_basis<<<blocks_for(count, kThreads), kThreads, 0, st>>>(s, count, index);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

namespace {

// How one marginal query reduces: the kernel family, its partial count and the
// workspace doubles the partials need beyond the handle scratch.
struct MargPlan {
  int kind = 0;        // 0 k_marg_low, 1 k_marg_thread, 2 k_marg_seg
  uint64_t parts = 1;  // blocks of k_marg_low / segments per output of k_marg_seg
  uint64_t work = 0;   // doubles of caller workspace (0: none needed)
  MargParams P{};
};

MargPlan plan_marginal(uint32_t n, const uint32_t* qubits, uint32_t k, int device) {
  MargPlan m;
  uint64_t mask = 0;
  for (uint32_t b = 0; b < k; ++b) {
    m.P.q[b] = qubits[b];
    mask |= 1ULL << qubits[b];
  }
  m.P.k = k;
  m.P.rest.np = 0;
  for (uint32_t b = 0; b < 64 && m.P.rest.np < 32; ++b)
    if (mask >> b & 1ULL) m.P.rest.p[m.P.rest.np++] = b;
  const uint64_t nj = 1ULL << k;
  const uint64_t nterms = 1ULL << (n - k);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint32_t top = k ? m.P.rest.p[m.P.rest.np - 1] : 0;  // highest marginal position
  if (k >= 1 && top < 10 && n >= 20 && nterms > 64) {
    // all marginal qubits in the low 10 bits (e.g. after a relabeling)
    uint64_t nb = 1;
    while (nb * 2 <= (uint64_t)sms * 4 && (1ULL << n) / (nb * 2) >= 1024 * 4) nb *= 2;
    m.kind = 0;
    m.parts = nb;
    m.work = nj * nb;
    return m;
  }
  // thread-per-output (exact reference order) when there are enough outputs
  // to fill the GPU or few terms per output
  if (nterms <= 64 || nj >= (uint64_t)sms * 1024) {
    m.kind = 1;
    return m;
  }
  // a power of two number of segments per output (dividing nterms), about
  // 8 blocks per SM in total, each segment at least one block's worth
  const uint64_t target_blocks = (uint64_t)sms * 8;
  uint64_t nseg = 1;
  while (nj * nseg * 2 <= target_blocks && nseg * 2 * kRedThreads <= nterms) nseg <<= 1;
  while (nj * nseg > (uint64_t)kPartials && nseg > 1) nseg >>= 1;
  m.kind = 2;
  m.parts = nseg;
  m.work = nj * nseg > (uint64_t)kPartials ? nj * nseg : 0;
  return m;
}

}  // namespace

uint64_t marginal_workspace(uint32_t n, const uint32_t* qubits, uint32_t k, int device) {
  return plan_marginal(n, qubits, k, device).work;
}

int launch_marginal(const double2* s, uint32_t n, const uint32_t* qubits, uint32_t k,
                    double* d_out, double* d_work, Scratch& sc, cudaStream_t st, int device) {
  const MargPlan m = plan_marginal(n, qubits, k, device);
  const uint64_t nj = 1ULL << k;
  double* tmp = nullptr;  // allocated here only when the caller gave no workspace
  double* work = d_work;
  if (m.work && !work) {
    DQ_CUDA_TRY(pool_malloc_async((void**)&tmp, sizeof(double) * m.work, st));
    work = tmp;
  }
  if (m.kind == 0) {
    k_marg_low<<<(unsigned)m.parts, 1024, 0, st>>>(s, (1ULL << n) / m.parts, m.P, work);
    k_marg_sum<<<blocks_for(nj, kThreads), kThreads, 0, st>>>(work, nj, (uint32_t)m.parts, d_out);
  } else if (m.kind == 1) {
    k_marg_thread<<<blocks_for(nj, kThreads), kThreads, 0, st>>>(s, nj, 1ULL << (n - k), m.P, d_out);
  } else {
    double* partial = m.work ? work : sc.d_partial;
    k_marg_seg<<<(unsigned)(nj * m.parts), kRedThreads, 0, st>>>(s, 1ULL << (n - k), (uint32_t)m.parts,
                                                                  m.P, partial);
    k_marg_sum<<<blocks_for(nj, kThreads), kThreads, 0, st>>>(partial, nj, (uint32_t)m.parts, d_out);
  }
  if (tmp) DQ_CUDA_TRY(cudaFreeAsync(tmp, st));
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

uint64_t cdf_workspace(uint64_t len) { return (len + kScanChunk - 1) / kScanChunk; }

int launch_cdf(double* d, uint64_t len, double* d_work, cudaStream_t st, int device) {
  (void)device;
  const uint64_t nb = cdf_workspace(len);
  double* tmp = nullptr;  // allocated here only when the caller gave no workspace
  double* sums = d_work;
  if (!sums) {
    DQ_CUDA_TRY(pool_malloc_async((void**)&tmp, sizeof(double) * nb, st));
    sums = tmp;
  }
  k_scan_sums<<<(unsigned)nb, kScanThreads, 0, st>>>(d, len, sums);
  k_scan_offsets<<<1, kScanThreads, 0, st>>>(sums, nb);
  k_scan_apply<<<(unsigned)nb, kScanThreads, 0, st>>>(d, len, sums);
  k_set_last_one<<<1, 1, 0, st>>>(d, len);
  if (tmp) DQ_CUDA_TRY(cudaFreeAsync(tmp, st));
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int launch_sample(const double* cdf, uint64_t len, const uint32_t key[8], uint64_t shots,
                  uint32_t* d_idx, unsigned long long* d_boundary, cudaStream_t st, int device) {
  (void)device;
  if (shots == 0) return DQ_OK;
  Key8 K;
  for (int i = 0; i < 8; ++i) K.k[i] = key[i];
  k_sample<<<blocks_for(shots, kThreads), kThreads, 0, st>>>(cdf, len, K, shots, d_idx, d_boundary);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

}  // namespace dq
