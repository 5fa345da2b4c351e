// dq_fused.cu — the tile-sweep engine: planner (host) and sweep kernel (sm_100a).
//
// The device side (tile geometry, the encoded program layout, the per-op
// register arithmetic and the per-CTA tile loop) is in dq_sweep.cuh.  The
// default launch runs 128 threads per CTA, three CTAs per SM.
//
// A sweep is a list of phases.  In a phase each thread holds 2^RB amplitudes
// in registers: the ones whose RB "register" local bits vary, at the thread
// bits given by its thread index.  Gate ops of the phase act on register
// bits only (dense 2x2 / 4x4, controlled X), so no data is exchanged between
// threads inside a phase; a new phase re-reads the tile with a new register
// assignment.  Per-gate arithmetic uses FMA (the tile path is held to the
// 1e-12 amplitude tolerance, the per-gate kernels to bit-exactness).
//
// Diagonal gates never need locality: they are accumulated on the host as a
// phase polynomial  c * prod_q w_q^{x_q} * prod_{q<r} w_qr^{x_q x_r}  and a
// FLUSH op applies all terms containing a qubit q right before the first
// non-diagonal gate on q.  A FLUSH multiplies the amplitudes with x_q = 1 by
// slot[s] * prod_{thread partners set} w * F[register index], where the
// per-tile factor slot[s] (q's linear term times its non-local partners
// whose bits are set in this tile's base index) is computed once per tile.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "dq_common.cuh"
#include "dq_fused.cuh"
#include "dq_gates.hpp"
#include "dq_sweep.cuh"

namespace dq {

namespace {

// One persistent CTA per SM walks tiles blockIdx.x, + gridDim.x, ...
// S = 1 (128 threads): no prefetch, three CTAs per SM overlap each other's
// loads.  S = 2: the next tile's load is in flight while the current one is
// computed.  The sweep program is staged in shared memory once per launch
// (read from global memory per op instead, QFT30 ran 38% slower).
// FORM_H (every phase an H phase) and FORM_U (plain one-qubit ops only): built
// without the generic op interpreter (FORM_U: with its one-qubit part only),
// in few enough registers for four CTAs per SM.
template <int TB, int RB, int S, int RUNB, int FORM = FORM_ALL>
__global__ void __launch_bounds__(1 << TB, (S == 1 && TB == 7 ? (FORM != FORM_ALL ? 4 : 3)
                                                              : (TB + RB <= 11 ? 2 : 1)))
    k_sweep(double2* __restrict__ state, const uint8_t* __restrict__ gprog, uint32_t prog_bytes,
            uint32_t ntiles, long long synth) {
  constexpr int T = 1 << (TB + RB);
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* bufs = reinterpret_cast<double2*>(smraw);  // S tiles
  double2* slots = bufs + S * T;
  uint8_t* sprog = reinterpret_cast<uint8_t*>(slots + kMaxSlots);
  for (uint32_t i = threadIdx.x * 16u; i < prog_bytes; i += (1u << TB) * 16u)
    *reinterpret_cast<uint4*>(sprog + i) = __ldg(reinterpret_cast<const uint4*>(gprog + i));
  __syncthreads();
  sweep_tiles<TB, RB, S, RUNB, FORM>(state, sprog, ntiles, synth, bufs, slots, blockIdx.x, gridDim.x);
}

// Sweep k of many states in one launch: job j's tiles are split into chunks
// of chunk_tiles consecutive tiles and the CTAs take (job, chunk) work items
// in order; a CTA stages a job's program in shared memory when it moves to
// that job (a few KB per chunk of 2 MB of tiles).
template <int TB, int RB, int RUNB, int FORM = FORM_ALL>
__global__ void __launch_bounds__(1 << TB, TB == 7 ? (FORM != FORM_ALL ? 4 : 3) : 2)
    k_sweep_multi(const SweepJob* __restrict__ jobs, uint32_t njobs, uint32_t nchunks,
                  uint32_t chunk_tiles, uint32_t ntiles) {
  constexpr int T = 1 << (TB + RB);
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* bufs = reinterpret_cast<double2*>(smraw);
  double2* slots = bufs + T;
  uint8_t* sprog = reinterpret_cast<uint8_t*>(slots + kMaxSlots);
  const uint64_t work = (uint64_t)njobs * nchunks;
  uint64_t staged = ~0ULL;
  for (uint64_t w = blockIdx.x; w < work; w += gridDim.x) {
    const uint64_t j = w / nchunks;
    const SweepJob J = jobs[j];
    if (j != staged) {
      for (uint32_t i = threadIdx.x * 16u; i < J.prog_bytes; i += (1u << TB) * 16u)
        *reinterpret_cast<uint4*>(sprog + i) = __ldg(reinterpret_cast<const uint4*>(J.prog + i));
      __syncthreads();
      staged = j;
    }
    const uint32_t c = (uint32_t)(w % nchunks);
    const uint32_t t0 = c * chunk_tiles;
    const uint32_t t1 = min(t0 + chunk_tiles, ntiles);
    sweep_tiles<TB, RB, 1, RUNB, FORM>(J.state, sprog, t1, J.synth, bufs, slots, t0, 1);
    __syncthreads();
  }
}

// ---- relabel materialisation: paired-tile involution of bit positions ------------
//
// A bit-position involution tau (tau(tau(p)) = p) moves amplitude i to tau(i).
// With a local set L closed under tau, tile T maps onto tile tau(T), element
// e onto tau_L(e); one CTA exchanges the pair (T, tau(T)) so the permutation
// is race-free in place.

struct PermParams {
  uint32_t m;             // |L|
  uint32_t L[kMaxM];      // local positions, ascending
  uint32_t tauL[kMaxM];   // local index of tau(L[k])
  uint32_t tau[64];       // tau on all positions
  uint32_t n;
};

__device__ __forceinline__ uint32_t perm_slot(uint32_t e) { return e + (e >> 4); }  // pad 1 per 16

__global__ void __launch_bounds__(256) k_permute_pairs(double2* __restrict__ state, PermParams P) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const uint32_t cnt = 1u << P.m;
  double2* A = reinterpret_cast<double2*>(smraw);
  double2* B = A + perm_slot(cnt);
  uint64_t bT = blockIdx.x;
  for (uint32_t k = 0; k < P.m; ++k) bT = insert_zero(bT, P.L[k]);
  uint64_t bU = 0;
  for (uint32_t p = 0; p < P.n; ++p)
    if ((bT >> p) & 1ULL) bU |= 1ULL << P.tau[p];
  if (bU < bT) return;  // the partner CTA handles this pair
  const bool self = (bU == bT);
  // element e of a tile: global offset dep(e)
  for (uint32_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    uint64_t d = 0;
    for (uint32_t k = 0; k < P.m; ++k)
      if ((e >> k) & 1u) d |= 1ULL << P.L[k];
    A[perm_slot(e)] = state[bT | d];
    if (!self) B[perm_slot(e)] = state[bU | d];
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    uint64_t d = 0;
    uint32_t te = 0;
    for (uint32_t k = 0; k < P.m; ++k)
      if ((e >> k) & 1u) {
        d |= 1ULL << P.L[k];
        te |= 1u << P.tauL[k];
      }
    // destination element e of tile U receives source element tau_L(e) of tile T
    state[bU | d] = A[perm_slot(te)];
    if (!self) state[bT | d] = B[perm_slot(te)];
  }
}

// =========================================================================
// host side: planner
// =========================================================================

inline hc conj(hc a) { return hc{a.re, -a.im}; }
inline bool is_unit_phase(hc a) { return fabs(a.re * a.re + a.im * a.im - 1.0) < 1e-12; }

enum PKind { PG_DIAG, PG_U1, PG_U1X, PG_U2 };

struct PGate {
  PKind kind = PG_DIAG;
  uint32_t t0 = 0, t1 = 0;  // physical targets (U2: t0 = MSB of the gate index)
  uint64_t ctrl = 0;        // physical controls (all must be 1)
  hc u[16];
  bool real = false;
  bool had = false;         // uncontrolled s*[[1,1],[1,-1]]: add/sub, scale deferred
  // diagonal terms
  hc cst{1, 0};
  int nlin = 0;
  uint32_t lq[2] = {0, 0};
  hc lw[2];
  bool quad = false;
  uint32_t qa = 0, qb = 0;
  hc qw{1, 0};
  uint64_t touched = 0;
};

struct Poly {
  uint32_t n = 0;
  std::vector<hc> lin;
  std::vector<char> hl;
  std::vector<hc> quad;
  std::vector<char> hq;
  std::vector<int> cnt;
  hc cst{1, 0};
  bool has_cst = false;

  void init(uint32_t nq) {
    n = nq;
    lin.assign(n, hc{1, 0});
    hl.assign(n, 0);
    quad.assign((size_t)n * n, hc{1, 0});
    hq.assign((size_t)n * n, 0);
    cnt.assign(n, 0);
    cst = hc{1, 0};
    has_cst = false;
  }
  void mul_lin(uint32_t q, hc w) {
    if (!hl[q]) { hl[q] = 1; ++cnt[q]; lin[q] = w; } else lin[q] = lin[q] * w;
  }
  void mul_quad(uint32_t a, uint32_t b, hc w) {
    const uint32_t lo = std::min(a, b), hi = std::max(a, b);
    const size_t k = (size_t)lo * n + hi;
    if (!hq[k]) { hq[k] = 1; ++cnt[lo]; ++cnt[hi]; quad[k] = w; } else quad[k] = quad[k] * w;
  }
  void add(const PGate& g) {
    if (!(g.cst.re == 1.0 && g.cst.im == 0.0)) { cst = cst * g.cst; has_cst = true; }
    for (int i = 0; i < g.nlin; ++i) mul_lin(g.lq[i], g.lw[i]);
    if (g.quad) mul_quad(g.qa, g.qb, g.qw);
  }
  bool pending(uint32_t q) const { return cnt[q] > 0; }
  bool empty() const {
    for (uint32_t q = 0; q < n; ++q)
      if (cnt[q]) return false;
    return true;
  }
  // remove and return all terms containing q
  void take(uint32_t q, hc* wlin, std::vector<std::pair<uint32_t, hc>>& partners) {
    *wlin = hl[q] ? lin[q] : hc{1, 0};
    if (hl[q]) { hl[q] = 0; --cnt[q]; lin[q] = hc{1, 0}; }
    partners.clear();
    for (uint32_t r = 0; r < n; ++r) {
      if (r == q) continue;
      const uint32_t lo = std::min(q, r), hi = std::max(q, r);
      const size_t k = (size_t)lo * n + hi;
      if (!hq[k]) continue;
      partners.push_back({r, quad[k]});
      hq[k] = 0;
      quad[k] = hc{1, 0};
      --cnt[q];
      --cnt[r];
    }
  }
};

struct POp {
  uint32_t type;
  int gate = -1;            // index into the segment's gate list
  uint32_t q = 0;           // FLUSH target (physical)
  hc wlin{1, 0};
  std::vector<std::pair<uint32_t, hc>> partners;   // FLUSH partners (physical)
  hc gcst{1, 0};                                  // GPHASE constant
  std::vector<std::pair<uint64_t, hc>> gterms;     // GPHASE per-tile terms (masks)
};

struct PSweep {
  std::vector<uint32_t> local;  // physical, ascending, size m
  std::vector<POp> ops;
};

// Blob writer (16-byte aligned sections)
struct Blob {
  std::vector<uint8_t> buf;
  size_t align16() {
    while (buf.size() % 16) buf.push_back(0);
    return buf.size();
  }
  template <class T>
  size_t put(const T* p, size_t count) {
    const size_t off = align16();
    const uint8_t* s = reinterpret_cast<const uint8_t*>(p);
    buf.insert(buf.end(), s, s + sizeof(T) * count);
    return off;
  }
};

struct Planner {
  uint32_t n = 0, M = 12, RB = 5, TB = 8;
  // FP64 work per amplitude one sweep may take on: at 30 qubits a sweep's
  // compute stays cheaper than another pass over the state up to ~100
  // (brickwork28 of u3 + cx: 255 ms at 48, 227 ms at 96, the same above)
  double budget = 96.0;
  uint32_t max_ops = 40;    // non-diagonal gates per sweep (bounds the staged program)
  bool single_tile = false;
  // qubits every tile holds (0..4: 512-byte runs; 0..2: 128-byte runs)
  uint64_t pinned = 0x1FULL;
  bool pin_auto = false;

  // cost in FP64 instructions per amplitude
  double gate_cost(const PGate& g) const {
    const double frac = 1.0 / (double)(1ULL << __builtin_popcountll(g.ctrl));
    switch (g.kind) {
      case PG_U1: return g.had ? 2.0 : (g.real ? 4.0 : 8.0) * frac;
      case PG_U1X: return 0.5;
      case PG_U2: return 16.0 * frac;
      default: return 0.0;
    }
  }

  static uint64_t targets(const PGate& g) {
    if (g.kind == PG_DIAG) return 0;
    if (g.kind == PG_U2) return (1ULL << g.t0) | (1ULL << g.t1);
    return 1ULL << g.t0;
  }

  // Split the gate list into sweeps; poly carries pending diagonal terms.
  void plan(std::vector<PGate>& G, Poly& poly, std::vector<PSweep>& out) {
    std::vector<int> rem(G.size());
    for (size_t i = 0; i < G.size(); ++i) rem[i] = (int)i;
    const uint64_t low_mask = single_tile ? ((n >= 64) ? ~0ULL : ((1ULL << n) - 1)) : pinned;
    while (!rem.empty()) {
      uint64_t S = low_mask;
      uint64_t blocked = 0;
      double cost = 0.0;
      std::vector<int> incl, next;
      bool any_nd = false;
      uint32_t nd_count = 0;
      uint64_t diag_touched = 0;
      // conservative size of the encoded program: op + matrix, and a flush
      // per target (op, lane/warp/register tables, slot and its non-local terms)
      size_t bytes = 4096 + 3072;
      const size_t flush_bytes = 48 + 16 * (32 + 8 + 16) + 32 + 32 * (size_t)n;
      for (int gi : rem) {
        const PGate& g = G[gi];
        if (g.touched & blocked) {
          next.push_back(gi);
          blocked |= g.touched;
          continue;
        }
        if (g.kind == PG_DIAG) {
          incl.push_back(gi);
          diag_touched |= g.touched;
          continue;
        }
        const uint64_t need = targets(g);
        const uint64_t ns = S | need;
        double c = gate_cost(g);
        uint64_t tm = need;
        while (tm) {
          const int t = __builtin_ctzll(tm);
          tm &= tm - 1;
          if (poly.pending((uint32_t)t) || ((diag_touched >> t) & 1ULL)) c += 4.0;  // a flush
        }
        const size_t gb = 48 + 16 * 16 + flush_bytes * (size_t)__builtin_popcountll(need);
        const bool fits = (uint32_t)__builtin_popcountll(ns) <= M && nd_count < max_ops &&
                          bytes + gb <= (size_t)max_prog((int)M) - 8192;
        const bool afford = single_tile || !any_nd || cost + c <= budget;
        if (!fits || !afford) {
          next.push_back(gi);
          blocked |= g.touched;
          continue;
        }
        S = ns;
        cost += c;
        bytes += gb;
        any_nd = true;
        ++nd_count;
        incl.push_back(gi);
      }
      // pad the local set to M qubits now: every later decision (which flush
      // partners are local, which per-tile terms test base bits) depends on it
      for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(S) < M; ++q) S |= 1ULL << q;
      PSweep sw;
      for (int gi : incl) {
        const PGate& g = G[gi];
        if (g.kind == PG_DIAG) {
          poly.add(g);
          continue;
        }
        uint64_t tm = targets(g);
        while (tm) {
          const uint32_t t = (uint32_t)__builtin_ctzll(tm);
          tm &= tm - 1;
          if (poly.pending(t)) {
            POp f;
            f.type = OP_FLUSH_R;
            f.q = t;
            poly.take(t, &f.wlin, f.partners);
            sw.ops.push_back(std::move(f));
          }
        }
        POp op;
        op.type = g.kind == PG_U1 ? (g.had ? OP_U1H : g.real ? OP_U1R : OP_U1)
                  : g.kind == PG_U1X ? OP_U1X : OP_U2;
        op.gate = gi;
        sw.ops.push_back(std::move(op));
      }
      for (uint32_t q = 0; q < n; ++q)
        if (S >> q & 1ULL) sw.local.push_back(q);
      out.push_back(std::move(sw));
      rem.swap(next);
    }
  }

  // Apply every pending term in the last sweep (appending one if needed).
  void final_flush(Poly& poly, std::vector<PSweep>& sweeps) {
    if (poly.empty() && !poly.has_cst) return;
    if (sweeps.empty()) {
      PSweep sw;
      uint64_t S = single_tile ? ((n >= 64) ? ~0ULL : ((1ULL << n) - 1)) : pinned;
      for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(S) < M; ++q)
        if (poly.pending(q)) S |= 1ULL << q;
      for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(S) < M; ++q) S |= 1ULL << q;
      for (uint32_t q = 0; q < n; ++q)
        if (S >> q & 1ULL) sw.local.push_back(q);
      sweeps.push_back(std::move(sw));
    }
    PSweep& last = sweeps.back();
    uint64_t S = 0;
    for (uint32_t q : last.local) S |= 1ULL << q;
    for (uint32_t q = 0; q < n; ++q) {
      if (!(S >> q & 1ULL) || !poly.pending(q)) continue;
      POp f;
      f.type = OP_FLUSH_T;  // resolved to R/T by the phase layout
      f.q = q;
      poly.take(q, &f.wlin, f.partners);
      last.ops.push_back(std::move(f));
    }
    // what is left involves non-local qubits only: a per-tile constant
    POp gp;
    gp.type = OP_GPHASE;
    gp.gcst = poly.has_cst ? poly.cst : hc{1, 0};
    for (uint32_t q = 0; q < n; ++q) {
      if (poly.hl[q]) gp.gterms.push_back({1ULL << q, poly.lin[q]});
      for (uint32_t r = q + 1; r < n; ++r) {
        const size_t k = (size_t)q * n + r;
        if (poly.hq[k]) gp.gterms.push_back({(1ULL << q) | (1ULL << r), poly.quad[k]});
      }
    }
    const bool trivial = gp.gterms.empty() && gp.gcst.re == 1.0 && gp.gcst.im == 0.0;
    if (!trivial) last.ops.push_back(std::move(gp));
    poly.init(n);
  }
};

// choose thread-bit order: lanes 0..2 need linearly independent swizzle vectors
bool order_thread_bits(std::vector<uint32_t>& tb) {
  const size_t c = tb.size();
  for (size_t i = 0; i < c; ++i)
    for (size_t j = i + 1; j < c; ++j)
      for (size_t k = j + 1; k < c; ++k) {
        const uint32_t a = swz_vec(tb[i]), b = swz_vec(tb[j]), d = swz_vec(tb[k]);
        if (a == b || (a ^ b) == 0 || d == a || d == b || d == (a ^ b)) continue;
        std::vector<uint32_t> o = {tb[i], tb[j], tb[k]};
        for (size_t x = 0; x < c; ++x)
          if (x != i && x != j && x != k) o.push_back(tb[x]);
        tb = o;
        return true;
      }
  return false;
}

// Encode a planned sweep into the device blob format.
int encode_sweep(const PSweep& sw_in, const std::vector<PGate>& G, uint32_t TBn, uint32_t RB,
                 Blob& blob, size_t* offset) {
  const int kSwTB = (int)TBn;
  const uint32_t m = (uint32_t)sw_in.local.size();
  if (m != kSwTB + RB) return fail(DQ_ERR_INTERNAL, "sweep local set size mismatch");
  int lidx[64];
  for (int i = 0; i < 64; ++i) lidx[i] = -1;
  for (uint32_t k = 0; k < m; ++k) lidx[sw_in.local[k]] = (int)k;

  // Uncontrolled X gates on local bits that no earlier op of the sweep
  // involves (as target or control; any flush or global phase stops the scan
  // for good) commute to the front of the sweep and fold into the tile load:
  // element e is stored at the shared-memory slot of e with those bits
  // flipped (the swizzled layout is XOR-linear), so they cost nothing.
  PSweep sw;
  sw.local = sw_in.local;
  uint32_t tile_xload = 0;
  {
    uint64_t involved = 0;
    bool stopped = false;
    for (const POp& op : sw_in.ops) {
      if (!stopped && op.type == OP_U1X && op.gate >= 0 && G[op.gate].ctrl == 0) {
        const uint32_t t = G[op.gate].t0;
        if (!((involved >> t) & 1ULL) && lidx[t] >= 0) {
          tile_xload ^= swz(1u << (uint32_t)lidx[t]);
          continue;
        }
      }
      if (op.type == OP_FLUSH_R || op.type == OP_FLUSH_T || op.type == OP_GPHASE) stopped = true;
      if (op.gate >= 0) involved |= (1ULL << G[op.gate].t0) | G[op.gate].ctrl |
                                    (op.type == OP_U2 ? (1ULL << G[op.gate].t1) : 0ULL);
      sw.ops.push_back(op);
    }
  }

  // phases: consecutive ops whose register needs fit RB register bits
  struct PhaseTmp {
    std::vector<uint32_t> regs;  // local bits
    size_t ob, oe;
  };
  std::vector<PhaseTmp> phases;
  auto need_of = [&](const POp& op, std::vector<uint32_t>& nd) {
    nd.clear();
    if (op.type == OP_U1 || op.type == OP_U1R || op.type == OP_U1X || op.type == OP_U1H) {
      nd.push_back((uint32_t)lidx[G[op.gate].t0]);
    } else if (op.type == OP_U2) {
      nd.push_back((uint32_t)lidx[G[op.gate].t0]);
      nd.push_back((uint32_t)lidx[G[op.gate].t1]);
    } else if (op.type == OP_FLUSH_R) {
      nd.push_back((uint32_t)lidx[op.q]);   // precedes the gate on q: same phase
    }
  };
  {
    size_t i = 0;
    std::vector<uint32_t> nd;
    while (i < sw.ops.size()) {
      PhaseTmp ph;
      ph.ob = i;
      size_t j = i;
      while (j < sw.ops.size()) {
        need_of(sw.ops[j], nd);
        std::vector<uint32_t> u = ph.regs;
        for (uint32_t b : nd)
          if (std::find(u.begin(), u.end(), b) == u.end()) u.push_back(b);
        if (u.size() > RB) break;
        ph.regs = u;
        ++j;
      }
      if (j == i) return fail(DQ_ERR_INTERNAL, "op needs more register bits than a phase has");
      ph.oe = j;
      phases.push_back(ph);
      i = j;
    }
    if (phases.empty()) phases.push_back(PhaseTmp{{}, 0, 0});
  }

  double scale = 1.0;  // product of the deferred Hadamard factors
  struct EncOp {
    uint32_t type = 0, b0 = 0, b1 = 0, creg = 0, ctl_thr = 0, flags = 0, slot = 0, data = 0;
    uint64_t cnl = 0;
  };
  std::vector<SwPhase> P;
  std::vector<EncOp> O;
  std::vector<SwSlot> SL;
  std::vector<SwSlotEnt> SE;
  std::vector<double2> D;
  auto d2 = [](hc z) { return make_double2(z.re, z.im); };
  auto add_slot = [&](hc w0, const std::vector<std::pair<uint64_t, hc>>& ents) -> uint32_t {
    SwSlot s{};
    s.count = (uint32_t)ents.size();
    s.start = (uint32_t)SE.size();
    s.w0 = d2(w0);
    for (auto& e : ents) {
      SwSlotEnt x{};
      x.mask = e.first;
      x.w = d2(e.second);
      SE.push_back(x);
    }
    SL.push_back(s);
    return (uint32_t)SL.size() - 1;
  };

  uint32_t carry_xload = 0;
  std::vector<uint32_t> last_tb, last_regs;  // thread / register bits of the last phase
  for (const PhaseTmp& ph : phases) {
    SwPhase sp{};
    // spare register slots take the highest unused local bits, so that the
    // lowest ones (qubits 0..2) stay thread bits: lanes 0..2 then cover
    // 128-byte runs, which the last phase's direct writes need
    std::vector<uint32_t> regs = ph.regs;
    for (uint32_t b = m; b-- > 0 && regs.size() < RB;)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
    std::vector<uint32_t> tb;
    for (uint32_t b = 0; b < m; ++b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) tb.push_back(b);
    if (tb.size() != (size_t)kSwTB || !order_thread_bits(tb))
      return fail(DQ_ERR_INTERNAL, "no bank-conflict-free thread layout");
    int rix[kMaxM], tix[kMaxM];
    for (int i = 0; i < kMaxM; ++i) rix[i] = tix[i] = -1;
    for (uint32_t b = 0; b < RB; ++b) { sp.V[b] = swz(1u << regs[b]); rix[regs[b]] = (int)b; }
    for (uint32_t b = RB; b < 4; ++b) sp.V[b] = 0;
    for (int i = 0; i < kSwTB; ++i) tix[tb[i]] = i;
    for (uint32_t ln = 0; ln < 32; ++ln) {
      uint32_t e = 0;
      for (int i = 0; i < 5; ++i)
        if ((ln >> i) & 1u) e |= 1u << tb[i];
      sp.lanesw[ln] = swz(e);
    }
    for (uint32_t wp = 0; wp < 8; ++wp) {
      uint32_t e = 0;
      for (int i = 0; i + 5 < kSwTB; ++i)
        if ((wp >> i) & 1u) e |= 1u << tb[5 + i];
      sp.warpsw[wp] = swz(e);
    }
    sp.op_begin = (uint32_t)O.size();
    // flush of a register target: per-tile slot, thread/register factor tables
    auto encode_flush = [&](const POp& op, EncOp& so) {
      const int l = lidx[op.q];
      std::vector<std::pair<uint64_t, hc>> nl;
      hc wthr[kMaxTB];
      for (int i = 0; i < kSwTB; ++i) wthr[i] = hc{1, 0};
      hc wreg[5];
      for (int i = 0; i < 5; ++i) wreg[i] = hc{1, 0};
      bool hasF = false;
      for (auto& pr : op.partners) {
        const int pl = lidx[pr.first];
        if (pl < 0) {
          nl.push_back({1ULL << pr.first, pr.second});
        } else if (rix[pl] >= 0) {
          wreg[rix[pl]] = wreg[rix[pl]] * pr.second;
          hasF = true;
        } else {
          wthr[tix[pl]] = wthr[tix[pl]] * pr.second;
        }
      }
      so.slot = add_slot(op.wlin, nl);
      const bool reg_target = rix[l] >= 0;
      bool thr = false;
      for (int i = 0; i < kSwTB; ++i)
        if (!(wthr[i].re == 1.0 && wthr[i].im == 0.0)) thr = true;
      if (thr) {
        so.flags |= FL_THR;
        for (uint32_t ln = 0; ln < 32; ++ln) {  // lane factor: thread bits 0..4
          hc f{1, 0};
          for (int i = 0; i < 5; ++i)
            if ((ln >> i) & 1u) f = f * wthr[i];
          D.push_back(d2(f));
        }
        for (uint32_t wp = 0; wp < 8; ++wp) {   // warp factor: thread bits 5..TB-1
          hc f{1, 0};
          for (int i = 0; i + 5 < kSwTB; ++i)
            if ((wp >> i) & 1u) f = f * wthr[5 + i];
          D.push_back(d2(f));
        }
      }
      if (hasF) {
        so.flags |= FL_REG;
        if (reg_target) {
          const uint32_t B = (uint32_t)rix[l];
          for (uint32_t idx = 0; idx < (1u << (RB - 1)); ++idx) {
            const uint32_t j = ((idx >> B) << (B + 1)) | (idx & ((1u << B) - 1));
            hc f{1, 0};
            for (uint32_t b = 0; b < RB; ++b)
              if (b != B && ((j >> b) & 1u)) f = f * wreg[b];
            D.push_back(d2(f));
          }
        } else {
          for (uint32_t j = 0; j < (1u << RB); ++j) {
            hc f{1, 0};
            for (uint32_t b = 0; b < RB; ++b)
              if ((j >> b) & 1u) f = f * wreg[b];
            D.push_back(d2(f));
          }
        }
      }
    };
    auto is_u1_type = [](uint32_t t) {
      return t == OP_U1 || t == OP_U1R || t == OP_U1X || t == OP_U1H;
    };
    // An uncontrolled X on a register bit that no earlier op of the phase
    // involves (as target, control or, conservatively, any flush) commutes to
    // the front of the phase and becomes part of the load: element j is read
    // from the address of j with that bit flipped (the swizzled addresses are
    // XOR-linear).  involved: register bits touched so far in this phase.
    uint32_t involved = 0;
    for (size_t oi = ph.ob; oi < ph.oe; ++oi) {
      const POp& op = sw.ops[oi];
      EncOp so{};
      so.type = op.type;
      // a flush of a register bit right before an uncontrolled one-qubit op on
      // the same qubit travels inside that op (FL_PRE)
      const POp* pre = nullptr;
      if ((op.type == OP_FLUSH_R || op.type == OP_FLUSH_T) && oi + 1 < ph.oe &&
          is_u1_type(sw.ops[oi + 1].type) && G[sw.ops[oi + 1].gate].ctrl == 0 &&
          G[sw.ops[oi + 1].gate].t0 == op.q && rix[lidx[op.q]] >= 0) {
        pre = &op;
        ++oi;
      }
      const POp& cur = sw.ops[oi];
      so.type = cur.type;
      if (!pre && cur.type == OP_U1X && G[cur.gate].ctrl == 0) {
        const uint32_t b = (uint32_t)rix[lidx[G[cur.gate].t0]];
        if (!((involved >> b) & 1u)) {
          sp.xload ^= sp.V[b];
          continue;
        }
      }
      if (pre || cur.type == OP_FLUSH_R || cur.type == OP_FLUSH_T || cur.type == OP_GPHASE)
        involved = ~0u;
      if (is_u1_type(cur.type) || cur.type == OP_U2) {
        const PGate& g = G[cur.gate];
        if (cur.type == OP_U1H) scale = scale * g.u[0].re;
        // controls: register bits, thread bits, non-local
        uint64_t cm = g.ctrl;
        while (cm) {
          const uint32_t c = (uint32_t)__builtin_ctzll(cm);
          cm &= cm - 1;
          const int l = lidx[c];
          if (l < 0) so.cnl |= 1ULL << c;
          else if (rix[l] >= 0) so.creg |= 1u << rix[l];
          else so.ctl_thr |= 1u << tix[l];
        }
        so.data = (uint32_t)D.size();
        if (cur.type == OP_U2) {
          int r0 = rix[lidx[g.t0]], r1 = rix[lidx[g.t1]];
          hc mm[16];
          for (int i = 0; i < 16; ++i) mm[i] = g.u[i];
          if (r0 > r1) {  // put the lower register bit first: swap the gate's index bits
            const int perm[4] = {0, 2, 1, 3};
            for (int r = 0; r < 4; ++r)
              for (int c = 0; c < 4; ++c) mm[r * 4 + c] = g.u[perm[r] * 4 + perm[c]];
            std::swap(r0, r1);
          }
          so.b0 = (uint32_t)r0;
          so.b1 = (uint32_t)r1;
          for (int i = 0; i < 16; ++i) D.push_back(d2(mm[i]));
        } else {
          so.b0 = (uint32_t)rix[lidx[g.t0]];
          for (int i = 0; i < 4; ++i) D.push_back(d2(g.u[i]));
          if (pre) {
            so.flags |= FL_PRE;
            encode_flush(*pre, so);
          }
        }
      } else if (cur.type == OP_FLUSH_R || cur.type == OP_FLUSH_T) {
        const int l = lidx[cur.q];
        so.data = (uint32_t)D.size();
        encode_flush(cur, so);
        if (rix[l] >= 0) {
          so.type = OP_FLUSH_R;
          so.b0 = (uint32_t)rix[l];
        } else {
          so.type = OP_FLUSH_T;
          so.b0 = (uint32_t)tix[l];
        }
      } else if (cur.type == OP_GPHASE) {
        so.slot = add_slot(cur.gcst, cur.gterms);
      }
      if (is_u1_type(cur.type)) involved |= (1u << so.b0) | so.creg;
      if (cur.type == OP_U2) involved |= (1u << so.b0) | (1u << so.b1) | so.creg;
      O.push_back(so);
    }
    if (&ph == &phases.back() && scale != 1.0) {
      // the deferred 1/sqrt(2) factors: fold into a per-tile phase if there is one
      bool folded = false;
      for (size_t oi = sp.op_begin; oi < O.size(); ++oi)
        if (O[oi].type == OP_GPHASE) {
          SL[O[oi].slot].w0.x *= scale;
          SL[O[oi].slot].w0.y *= scale;
          folded = true;
          break;
        }
      if (!folded) {
        EncOp so{};
        so.type = OP_SCALE;
        so.data = (uint32_t)D.size();
        D.push_back(make_double2(scale, 0.0));
        O.push_back(so);
      }
    }
    // A phase made only of uncontrolled Hadamard-pattern ops on register bits
    // 0, 1, ..., K-1 in that order (register bits are assigned in the order
    // the phase's ops need them), optionally followed by the deferred scale,
    // runs as straight-line code: an OP_HPHASE marker goes in front of them.
    {
      const size_t ob = sp.op_begin, oe = O.size();
      size_t k = 0;
      bool ok = oe > ob, sc = false;
      for (size_t i = ob; i < oe && ok; ++i) {
        const EncOp& x = O[i];
        if (x.type == OP_SCALE && i + 1 == oe && i > ob) {
          sc = true;
          continue;
        }
        ok = (x.type == OP_U1H || x.type == OP_U1R) && x.creg == 0 && x.ctl_thr == 0 && x.cnl == 0 &&
             x.b0 == (uint32_t)k;
        ++k;
      }
      // the deferred scale folds into the last op, which must then be a Hadamard
      if (sc && k >= 1 && O[ob + k - 1].type != OP_U1H) ok = false;
      if (ok && k >= 1 && k <= RB) {
        for (size_t i = ob; i < ob + k; ++i) {
          EncOp& x = O[i];
          if (!(x.flags & FL_PRE) || !(x.flags & FL_REG)) continue;
          // register-partner table entries equal to the entry of their low bits
          // (after the op's 4 matrix entries and, with FL_THR, its 40 thread factors)
          const size_t f0 = x.data + 4 + ((x.flags & FL_THR) ? 40 : 0);
          const uint32_t lowmask = (1u << x.b0) - 1u;
          bool low = true;
          for (uint32_t idx = 0; idx < (1u << (RB - 1)) && low; ++idx) {
            const double2 u = D[f0 + idx], v = D[f0 + (idx & lowmask)];
            low = u.x == v.x && u.y == v.y;
          }
          if (low) x.flags |= FL_LOWF;
        }
        EncOp hp{};
        hp.type = OP_HPHASE;
        hp.b1 = (uint32_t)k;
        hp.flags = sc ? HPH_SCALE : 0u;
        hp.data = sc ? O[oe - 1].data : 0u;
        O.insert(O.begin() + (ptrdiff_t)ob, hp);
      }
    }
    sp.op_end = (uint32_t)O.size();
    sp.xload ^= carry_xload;
    carry_xload = 0;
    if (sp.op_end == sp.op_begin && &ph != &phases.back()) {
      // no op left (all folded): its flips move to the next phase's load
      carry_xload = sp.xload;
      continue;
    }
    last_tb = tb;
    last_regs = regs;
    P.push_back(sp);
  }
  if (SL.size() > (size_t)kMaxSlots) return fail(DQ_ERR_INTERNAL, "too many per-tile slots");

  for (const SwPhase& sp : P) {
    for (int i = 0; i < 32; ++i)
      if (sp.lanesw[i] >= (1u << m)) return fail(DQ_ERR_INTERNAL, "thread index outside the tile");
    for (int i = 0; i < 8; ++i)
      if (sp.warpsw[i] >= (1u << m)) return fail(DQ_ERR_INTERNAL, "thread index outside the tile");
    for (uint32_t b = 0; b < RB; ++b)
      if (sp.V[b] >= (1u << m)) return fail(DQ_ERR_INTERNAL, "register bit outside the tile");
  }
  for (const EncOp& so : O)
    if (((so.type <= OP_U2 || so.type == OP_U1H || so.type == OP_FLUSH_R) && so.b0 >= RB) ||
        (so.type == OP_FLUSH_T && so.b0 >= (uint32_t)kSwTB) || (so.type == OP_U2 && so.b1 >= RB) ||
        so.slot >= SL.size() + (SL.empty() ? 1 : 0) || so.data > D.size() || so.slot > 0xffffu ||
        so.creg > 0xffu || so.ctl_thr > 0xffu || so.flags > 0xffu)
      return fail(DQ_ERR_INTERNAL, "op encoding out of range");
  std::vector<SwOp> OP(O.size());
  for (size_t i = 0; i < O.size(); ++i) {
    const EncOp& e = O[i];
    OP[i].w0 = e.type | (e.b0 << 8) | (e.b1 << 16) | (e.creg << 24);
    OP[i].w1 = e.ctl_thr | (e.flags << 8) | (e.slot << 16);
    OP[i].data = e.data;
    OP[i].cnl = e.cnl;
  }
  SwHeader h{};
  h.m = m;
  h.rb = RB;
  // runs of 2^run_bits: the sweep's lowest run_bits local bits are qubits 0..run_bits-1
  uint32_t run_bits = 0;
  while (run_bits < 5 && run_bits < m && sw.local[run_bits] == run_bits) ++run_bits;
  run_bits = run_bits >= 5 ? 5u : 3u;
  if (m < run_bits || sw.local[run_bits - 1] != run_bits - 1)
    return fail(DQ_ERR_INTERNAL, "sweep local set lacks the pinned low qubits");
  h.run_bits = run_bits;
  const uint32_t nruns = 1u << (m - run_bits);
  std::vector<uint64_t> runoff(nruns);
  std::vector<uint32_t> runswz(nruns);
  for (uint32_t r = 0; r < nruns; ++r) {
    uint64_t off = 0;
    for (uint32_t b = 0; b + run_bits < m; ++b)
      if ((r >> b) & 1u) off |= 1ULL << sw.local[run_bits + b];
    runoff[r] = off;
    runswz[r] = swz(r << run_bits);
  }
  h.nphase = (uint32_t)P.size();
  h.nslots = (uint32_t)SL.size();
  {
    // every phase a straight-line phase: Hadamard-pattern sub-ops only, or
    // real 2x2 sub-ops only, select a restricted build
    bool marked = !P.empty(), had = false, real = false;
    for (const SwPhase& sp : P)
      if (sp.op_begin >= sp.op_end || O[sp.op_begin].type != OP_HPHASE) marked = false;
    for (const EncOp& e : O) {
      had = had || e.type == OP_U1H;
      real = real || e.type == OP_U1R;
    }
    const bool honly = marked && !real;
    h.flags = honly ? SWF_HONLY : (marked && !had ? SWF_RONLY : 0u);
    bool uonly = !P.empty() && !marked;
    for (const EncOp& e : O)
      if (!(e.type == OP_U1 || e.type == OP_U1R || e.type == OP_U1X) || (e.flags & FL_PRE)) uonly = false;
    if (uonly) h.flags |= SWF_UONLY;
  }
  h.tile_xload = tile_xload;
  for (uint32_t k = 0; k < m; ++k) h.local_pos[k] = sw.local[k];
  const size_t hoff = blob.put(&h, 1);
  const size_t po = blob.put(P.data(), P.size());
  const size_t oo = OP.empty() ? blob.align16() : blob.put(OP.data(), OP.size());
  const size_t so = SL.empty() ? blob.align16() : blob.put(SL.data(), SL.size());
  const size_t eo = SE.empty() ? blob.align16() : blob.put(SE.data(), SE.size());
  const size_t dd = D.empty() ? blob.align16() : blob.put(D.data(), D.size());
  const size_t ro = blob.put(runoff.data(), runoff.size());
  const size_t rs = blob.put(runswz.data(), runswz.size());
  // The last phase writes straight to the state when its lanes 0..2 are local
  // bits 0..2 (qubits 0..2): every 8-lane group then writes one 128-byte run.
  size_t go = 0;
  if (!P.empty() && last_tb.size() >= 3 && last_tb[0] == 0 && last_tb[1] == 1 && last_tb[2] == 2 &&
      sw.local[0] == 0 && sw.local[1] == 1 && sw.local[2] == 2) {
    SwGStore g{};
    for (uint32_t ln = 0; ln < 32; ++ln)
      for (int i = 0; i < 5; ++i)
        if ((ln >> i) & 1u) g.glane[ln] |= 1ULL << sw.local[last_tb[i]];
    for (uint32_t wp = 0; wp < 8; ++wp)
      for (int i = 0; i + 5 < kSwTB; ++i)
        if ((wp >> i) & 1u) g.gwarp[wp] |= 1ULL << sw.local[last_tb[5 + i]];
    for (uint32_t b = 0; b < RB && b < 4; ++b) g.gV[b] = 1ULL << sw.local[last_regs[b]];
    go = blob.put(&g, 1);
  }
  SwHeader* hp = reinterpret_cast<SwHeader*>(blob.buf.data() + hoff);
  hp->off_runoff = (uint32_t)(ro - hoff);
  hp->off_runswz = (uint32_t)(rs - hoff);
  hp->off_gstore = go ? (uint32_t)(go - hoff) : 0u;
  hp->off_phase = (uint32_t)(po - hoff);
  hp->off_op = (uint32_t)(oo - hoff);
  hp->off_slot = (uint32_t)(so - hoff);
  hp->off_slotent = (uint32_t)(eo - hoff);
  hp->off_data = (uint32_t)(dd - hoff);
  blob.align16();
  hp = reinterpret_cast<SwHeader*>(blob.buf.data() + hoff);
  hp->prog_bytes = (uint32_t)(blob.buf.size() - hoff);
  if (hp->prog_bytes > (uint32_t)max_prog((int)m)) return fail(DQ_ERR_INTERNAL, "sweep program too large");
  *offset = hoff;
  return DQ_OK;
}

// ---- gate conversion ----------------------------------------------------------------

// Convert one instruction (logical qubits mapped through perm) into planner
// gates.  Returns false if the fused path cannot represent it.
bool convert_inst(const dq_inst& in, const uint32_t* perm, std::vector<PGate>& out,
                  uint32_t* swap_a, uint32_t* swap_b, bool* is_swap) {
  *is_swap = false;
  hc u[4];
  auto diag1 = [&](uint32_t t, hc u00, hc u11, uint64_t ctrl) -> bool {
    // diag(u00, u11) on t with <= 1 control; returns false for more controls
    PGate g;
    g.kind = PG_DIAG;
    const int nc = __builtin_popcountll(ctrl);
    if (nc > 1 || !is_unit_phase(u00) || !is_unit_phase(u11)) return false;
    const hc rel = (u00.re == 1.0 && u00.im == 0.0) ? u11 : u11 * conj(u00);
    if (nc == 0) {
      if (!(u00.re == 1.0 && u00.im == 0.0)) g.cst = u00;
      g.nlin = 1;
      g.lq[0] = t;
      g.lw[0] = rel;
      g.touched = 1ULL << t;
    } else {
      const uint32_t c = (uint32_t)__builtin_ctzll(ctrl);
      if (!(u00.re == 1.0 && u00.im == 0.0)) {
        g.nlin = 1;
        g.lq[0] = c;
        g.lw[0] = u00;
      }
      g.quad = true;
      g.qa = c;
      g.qb = t;
      g.qw = rel;
      g.touched = (1ULL << t) | ctrl;
    }
    out.push_back(g);
    return true;
  };
  auto u1 = [&](uint32_t t, const hc* m, uint64_t ctrl, bool xperm) {
    PGate g;
    g.kind = xperm ? PG_U1X : PG_U1;
    g.t0 = t;
    g.ctrl = ctrl;
    for (int i = 0; i < 4; ++i) g.u[i] = m[i];
    g.real = !xperm && m[0].im == 0.0 && m[1].im == 0.0 && m[2].im == 0.0 && m[3].im == 0.0;
    g.had = g.real && ctrl == 0 && m[0].re == m[1].re && m[0].re == m[2].re &&
            m[0].re == -m[3].re;
    g.touched = (1ULL << t) | ctrl;
    out.push_back(g);
  };
  if (matrix_1q(in.kind, in.p, u)) {
    const uint32_t t = perm[in.q[0]];
    if (is_zero(u[1]) && is_zero(u[2]) && diag1(t, u[0], u[3], 0)) return true;
    const bool xp = is_zero(u[0]) && is_zero(u[3]) && is_one(u[1]) && is_one(u[2]);
    u1(t, u, 0, xp);
    return true;
  }
  Gate g;
  if (!matrix_nq(in, g)) return false;
  for (uint32_t b = 0; b < g.k; ++b) g.qubits[b] = perm[g.qubits[b]];
  GateOp op;
  classify(g, op);
  switch (op.cls) {
    case GC_PHASE: {
      const hc one{1, 0};
      if (__builtin_popcountll(op.ctrl_mask) <= 1 && diag1(op.target, one, op.u[0], op.ctrl_mask))
        return true;
      hc m[4] = {one, hc{0, 0}, hc{0, 0}, op.u[0]};
      u1(op.target, m, op.ctrl_mask, false);
      return true;
    }
    case GC_ONE_Q:
      if (is_zero(op.u[1]) && is_zero(op.u[2]) && __builtin_popcountll(op.ctrl_mask) <= 1 &&
          diag1(op.target, op.u[0], op.u[3], op.ctrl_mask))
        return true;
      u1(op.target, op.u, op.ctrl_mask, false);
      return true;
    case GC_XPERM: {
      hc m[4] = {hc{0, 0}, hc{1, 0}, hc{1, 0}, hc{0, 0}};
      u1(op.target, m, op.ctrl_mask, true);
      return true;
    }
    case GC_SWAP: {
      if (op.ctrl_mask == 0) {
        *is_swap = true;
        // logical qubits of the swap (relabel the logical -> physical map)
        *swap_a = (uint32_t)in.q[in.nq - 2];
        *swap_b = (uint32_t)in.q[in.nq - 1];
        return true;
      }
      // controlled swap = cx(b->a) . ccx(c, a -> b) . cx(b->a), exact permutations
      const uint32_t a = op.target, b = op.target2;
      hc xm[4] = {hc{0, 0}, hc{1, 0}, hc{1, 0}, hc{0, 0}};
      u1(a, xm, (1ULL << b), true);
      u1(b, xm, op.ctrl_mask | (1ULL << a), true);
      u1(a, xm, (1ULL << b), true);
      return true;
    }
    case GC_DIAG: {
      if (g.k != 2) return false;
      const hc d00 = g.m[0], d01 = g.m[5], d10 = g.m[10], d11 = g.m[15];
      if (!is_unit_phase(d00) || !is_unit_phase(d01) || !is_unit_phase(d10) || !is_unit_phase(d11))
        return false;
      PGate p;
      p.kind = PG_DIAG;
      const uint32_t qa = g.qubits[0], qb = g.qubits[1];
      p.cst = d00;
      p.nlin = 2;
      p.lq[0] = qa;
      p.lw[0] = d10 * conj(d00);
      p.lq[1] = qb;
      p.lw[1] = d01 * conj(d00);
      p.quad = true;
      p.qa = qa;
      p.qb = qb;
      p.qw = d11 * d00 * conj(d01) * conj(d10);
      p.touched = (1ULL << qa) | (1ULL << qb);
      out.push_back(p);
      return true;
    }
    case GC_DENSE: {
      if (g.k != 2) return false;
      PGate p;
      p.kind = PG_U2;
      p.t0 = g.qubits[0];
      p.t1 = g.qubits[1];
      for (int i = 0; i < 16; ++i) p.u[i] = g.m[i];
      p.touched = (1ULL << p.t0) | (1ULL << p.t1);
      out.push_back(p);
      return true;
    }
    default:
      return false;
  }
}

template <int TB, int RB, int S, int RUNB, int FORM = FORM_ALL>
int launch_sweep_r(double2* amp, uint32_t n, const uint8_t* dblob, uint32_t prog_bytes,
                   cudaStream_t st, long long synth) {
  constexpr int M = TB + RB;
  const size_t smem_max = sizeof(double2) * (S * (1u << M) + kMaxSlots) + max_prog(M);
  const size_t smem = sizeof(double2) * (S * (1u << M) + kMaxSlots) + prog_bytes;
  // per device, once: opt-in shared memory; resident CTAs per SM for this
  // launch's shared memory (programs are mostly far below the maximum), cached
  // per 4 KB of program size (the mutex makes concurrent host threads safe)
  static std::mutex mu;
  static bool attr_done[64];
  static int per_sm[64][17];  // 0 = not yet queried
  int dev = 0;
  DQ_CUDA_TRY(cudaGetDevice(&dev));
  int resident;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_done[dev & 63]) {
      DQ_CUDA_TRY(cudaFuncSetAttribute(k_sweep<TB, RB, S, RUNB, FORM>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
      attr_done[dev & 63] = true;
    }
    const uint32_t bucket = std::min<uint32_t>(16, (prog_bytes + 4095) / 4096);
    const size_t smem_b = std::min(smem_max, smem - prog_bytes + 4096 * (size_t)bucket);
    int& r = per_sm[dev & 63][bucket];
    if (r == 0) {
      int b = 1;
      DQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep<TB, RB, S, RUNB, FORM>,
                                                                1 << TB, smem_b));
      r = b < 1 ? 1 : b;
    }
    resident = r;
  }
  int sms = 148;
  DQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint64_t tiles = 1ULL << (n - M);
  const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sms * resident);
  k_sweep<TB, RB, S, RUNB, FORM><<<grid, 1 << TB, smem, st>>>(amp, dblob, prog_bytes, (uint32_t)tiles,
                                                               synth);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

template <int TB, int RB>
int launch_sweep_rb(double2* amp, uint32_t n, const uint8_t* dblob, uint32_t prog_bytes,
                    cudaStream_t st, long long synth, uint32_t run_bits, uint32_t flags) {
  // default: single-buffered tiles, three 128-thread CTAs per SM (measured
  // faster than two double-buffered CTAs: the extra warps hide more of the
  // per-op latency than the prefetch saves); DQSIM_SWEEP_STAGES=2 selects
  // double buffering
  static const int stages = [] {
    const char* e = getenv("DQSIM_SWEEP_STAGES");
    return e ? atoi(e) : 1;
  }();
  if (TB == 7 && stages != 2) {
    if (RB == 4 && (flags & SWF_HONLY))
      return run_bits == 3 ? launch_sweep_r<7, 4, 1, 3, FORM_H>(amp, n, dblob, prog_bytes, st, synth)
                           : launch_sweep_r<7, 4, 1, 5, FORM_H>(amp, n, dblob, prog_bytes, st, synth);
    if (RB == 4 && (flags & SWF_RONLY))
      return run_bits == 3 ? launch_sweep_r<7, 4, 1, 3, FORM_R>(amp, n, dblob, prog_bytes, st, synth)
                           : launch_sweep_r<7, 4, 1, 5, FORM_R>(amp, n, dblob, prog_bytes, st, synth);
    if (RB == 4 && (flags & SWF_UONLY))
      return run_bits == 3 ? launch_sweep_r<7, 4, 1, 3, FORM_U>(amp, n, dblob, prog_bytes, st, synth)
                           : launch_sweep_r<7, 4, 1, 5, FORM_U>(amp, n, dblob, prog_bytes, st, synth);
    return run_bits == 3 ? launch_sweep_r<7, RB, 1, 3>(amp, n, dblob, prog_bytes, st, synth)
                         : launch_sweep_r<7, RB, 1, 5>(amp, n, dblob, prog_bytes, st, synth);
  }
  return run_bits == 3 ? launch_sweep_r<TB, RB, 2, 3>(amp, n, dblob, prog_bytes, st, synth)
                       : launch_sweep_r<TB, RB, 2, 5>(amp, n, dblob, prog_bytes, st, synth);
}

int launch_sweep(double2* amp, uint32_t n, uint32_t TB, uint32_t RB, const uint8_t* dblob,
                 uint32_t prog_bytes, cudaStream_t st, long long synth, uint32_t run_bits,
                 uint32_t flags) {
  if (TB == 8) {
    switch (RB) {
      case 2: return launch_sweep_rb<8, 2>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      case 3: return launch_sweep_rb<8, 3>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      case 4: return launch_sweep_rb<8, 4>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      default: break;
    }
  } else if (TB == 7) {
    switch (RB) {
      case 2: return launch_sweep_rb<7, 2>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      case 3: return launch_sweep_rb<7, 3>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      case 4: return launch_sweep_rb<7, 4>(amp, n, dblob, prog_bytes, st, synth, run_bits, flags);
      default: break;
    }
  }
  return fail(DQ_ERR_INTERNAL, "unsupported sweep geometry");
}

template <int TB, int RB, int RUNB, int FORM = FORM_ALL>
int launch_sweep_multi_t(const SweepJob* d_jobs, uint32_t njobs, uint32_t n, uint32_t max_bytes,
                         cudaStream_t st) {
  constexpr int M = TB + RB;
  const size_t smem_max = sizeof(double2) * ((1u << M) + kMaxSlots) + max_prog(M);
  const size_t smem = sizeof(double2) * ((1u << M) + kMaxSlots) + max_bytes;
  // resident CTAs per SM for this launch's shared memory, cached per 4 KB of
  // program size (programs are mostly far below the maximum)
  static std::mutex mu;
  static bool attr_done[64];
  static int per_sm[64][17];
  int dev = 0;
  DQ_CUDA_TRY(cudaGetDevice(&dev));
  int resident;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_done[dev & 63]) {
      DQ_CUDA_TRY(cudaFuncSetAttribute(k_sweep_multi<TB, RB, RUNB, FORM>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
      attr_done[dev & 63] = true;
    }
    const uint32_t bucket = std::min<uint32_t>(16, (max_bytes + 4095) / 4096);
    const size_t smem_b = std::min(smem_max, smem - max_bytes + 4096 * (size_t)bucket);
    int& r = per_sm[dev & 63][bucket];
    if (r == 0) {
      int b = 1;
      DQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep_multi<TB, RB, RUNB, FORM>,
                                                                1 << TB, smem_b));
      r = b < 1 ? 1 : b;
    }
    resident = r;
  }
  int sms = 148;
  DQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint32_t ntiles = 1u << (n - M);
  const uint32_t chunk = std::min<uint32_t>(64, ntiles);
  const uint32_t nchunks = (ntiles + chunk - 1) / chunk;
  const uint64_t work = (uint64_t)njobs * nchunks;
  const unsigned grid = (unsigned)std::min<uint64_t>(work, (uint64_t)sms * resident);
  k_sweep_multi<TB, RB, RUNB, FORM><<<grid, 1 << TB, smem, st>>>(d_jobs, njobs, nchunks, chunk, ntiles);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

int ensure_capacity(FusedWork& fw, size_t bytes, cudaStream_t st) {
  if (bytes <= fw.d_cap && bytes <= fw.h_cap) return DQ_OK;
  DQ_CUDA_TRY(cudaStreamSynchronize(st));
  size_t cap = std::max<size_t>(bytes, 1 << 16);
  cap = std::max(cap, fw.d_cap * 2);
  if (fw.d_blob) cudaFree(fw.d_blob);
  if (fw.h_blob) cudaFreeHost(fw.h_blob);
  fw.d_blob = nullptr;
  fw.h_blob = nullptr;
  fw.d_cap = fw.h_cap = 0;
  DQ_CUDA_TRY(cudaMalloc((void**)&fw.d_blob, cap));
  DQ_CUDA_TRY(cudaMallocHost((void**)&fw.h_blob, cap));
  fw.d_cap = fw.h_cap = cap;
  return DQ_OK;
}

}  // namespace

void fused_release(FusedWork& fw) {
  if (fw.d_blob) cudaFree(fw.d_blob);
  if (fw.h_blob) cudaFreeHost(fw.h_blob);
  for (auto e : fw.events) cudaEventDestroy(e);
  fw = FusedWork();
}

// ---- relabel materialisation ------------------------------------------------------------

int materialize_perm(double2* amp, uint32_t n, uint32_t* perm, cudaStream_t st, uint64_t* launches) {
  // sigma(p) = logical qubit stored at physical p: data bit p moves to sigma(p)
  uint32_t sigma[64];
  bool ident = true;
  for (uint32_t l = 0; l < n; ++l) {
    sigma[perm[l]] = l;
    if (perm[l] != l) ident = false;
  }
  if (ident) return DQ_OK;
  // sigma = tau2 o tau1, both involutions (cycle reflections)
  uint32_t tau1[64], tau2[64];
  for (uint32_t p = 0; p < n; ++p) tau1[p] = tau2[p] = p;
  std::vector<char> seen(n, 0);
  for (uint32_t p = 0; p < n; ++p) {
    if (seen[p]) continue;
    std::vector<uint32_t> cyc;
    uint32_t x = p;
    while (!seen[x]) {
      seen[x] = 1;
      cyc.push_back(x);
      x = sigma[x];
    }
    const size_t k = cyc.size();
    for (size_t i = 0; i < k; ++i) {
      tau1[cyc[i]] = cyc[(k - i) % k];
      tau2[cyc[i]] = cyc[(k + 1 - i) % k];
    }
  }
  const uint32_t* taus[2] = {tau1, tau2};
  for (int r = 0; r < 2; ++r) {
    const uint32_t* tau = taus[r];
    bool id = true;
    for (uint32_t p = 0; p < n; ++p)
      if (tau[p] != p) id = false;
    if (id) continue;
    // local set: closed under tau, contains 0..4 (or everything for small n)
    uint64_t L = 0;
    const uint32_t want = std::min<uint32_t>(n, 11);
    for (uint32_t p = 0; p < std::min<uint32_t>(n, 5); ++p) L |= (1ULL << p) | (1ULL << tau[p]);
    for (uint32_t p = 0; p < n && (uint32_t)__builtin_popcountll(L) < want; ++p) {
      if (L >> p & 1ULL) continue;
      const uint64_t add = (1ULL << p) | (1ULL << tau[p]);
      if ((uint32_t)__builtin_popcountll(L | add) <= (uint32_t)kMaxM) L |= add;
    }
    PermParams P{};
    P.n = n;
    P.m = 0;
    int li[64];
    for (uint32_t p = 0; p < n; ++p) {
      P.tau[p] = tau[p];
      li[p] = -1;
      if (L >> p & 1ULL) {
        li[p] = (int)P.m;
        P.L[P.m++] = p;
      }
    }
    for (uint32_t k = 0; k < P.m; ++k) P.tauL[k] = (uint32_t)li[tau[P.L[k]]];
    const size_t smem = sizeof(double2) * 2 * ((1u << P.m) + ((1u << P.m) >> 4));
    static std::mutex mu;
    static uint64_t attr_done = 0;  // one bit per device
    int dev = 0;
    DQ_CUDA_TRY(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> lk(mu);
      if (!((attr_done >> (dev & 63)) & 1ULL)) {
        DQ_CUDA_TRY(cudaFuncSetAttribute(k_permute_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(double2) * 2 * (4096 + 256))));
        attr_done |= 1ULL << (dev & 63);
      }
    }
    const uint64_t tiles = 1ULL << (n - P.m);
    k_permute_pairs<<<(unsigned)tiles, 256, smem, st>>>(amp, P);
    DQ_CUDA_TRY(cudaGetLastError());
    if (launches) ++*launches;
  }
  for (uint32_t l = 0; l < n; ++l) perm[l] = l;
  return DQ_OK;
}

// ---- program runner ------------------------------------------------------------------------

int fused_run_segment(double2* amp, uint32_t n, std::vector<PGate>& G, Planner& pl, Poly& poly,
                      FusedWork& fw, cudaStream_t st, bool timing, dq_profile* prof,
                      int64_t* lazy_basis) {
  std::vector<PSweep> sweeps;
  if (pl.pin_auto && !pl.single_tile) {
    // plan with qubits 0..4 pinned and with 0..2 pinned; the wider tile
    // choice wins only when it saves at least a tenth of the sweeps (its
    // 128-byte runs cost a little more per sweep)
    Poly poly3 = poly;
    std::vector<PSweep> sweeps3;
    pl.pinned = 0x1FULL;
    pl.plan(G, poly, sweeps);
    pl.final_flush(poly, sweeps);
    pl.pinned = 0x7ULL;
    pl.plan(G, poly3, sweeps3);
    pl.final_flush(poly3, sweeps3);
    if (10 * sweeps3.size() <= 9 * sweeps.size()) {
      sweeps.swap(sweeps3);
      poly = poly3;
    }
  } else {
    pl.plan(G, poly, sweeps);
    pl.final_flush(poly, sweeps);
  }
  if (sweeps.empty()) return DQ_OK;
  Blob blob;
  std::vector<size_t> offs(sweeps.size());
  for (size_t i = 0; i < sweeps.size(); ++i)
    DQ_TRY(encode_sweep(sweeps[i], G, pl.TB, pl.RB, blob, &offs[i]));
  blob.align16();
  if (fw.plan_out) {  // plan-only: hand the programs back instead of running them
    const size_t base = fw.plan_out->size();
    fw.plan_out->insert(fw.plan_out->end(), blob.buf.begin(), blob.buf.end());
    for (size_t o : offs) fw.plan_offs->push_back(base + o);
    fw.plan_rb = pl.RB;
    if (lazy_basis && *lazy_basis >= 0) {  // the first sweep generates the basis vector
      fw.plan_synth = *lazy_basis;
      *lazy_basis = -1;
    }
    prof->sweeps += sweeps.size();
    return DQ_OK;
  }
  // the pinned staging buffer may still feed an earlier copy
  DQ_CUDA_TRY(cudaStreamSynchronize(st));
  DQ_TRY(ensure_capacity(fw, blob.buf.size(), st));
  memcpy(fw.h_blob, blob.buf.data(), blob.buf.size());
  DQ_CUDA_TRY(cudaMemcpyAsync(fw.d_blob, fw.h_blob, blob.buf.size(), cudaMemcpyHostToDevice, st));
  for (size_t i = 0; i < sweeps.size(); ++i) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventRecord(e0, st);
    }
    const SwHeader* hh = reinterpret_cast<const SwHeader*>(blob.buf.data() + offs[i]);
    // a pending basis state is consumed by the first sweep (it writes every amplitude)
    const long long synth = (lazy_basis && *lazy_basis >= 0) ? (long long)*lazy_basis : -1;
    DQ_TRY(launch_sweep(amp, n, pl.TB, pl.RB, fw.d_blob + offs[i], hh->prog_bytes, st, synth,
                        hh->run_bits, hh->flags));
    if (lazy_basis) *lazy_basis = -1;
    if (timing) {
      cudaEventRecord(e1, st);
      fw.events.push_back(e0);
      fw.events.push_back(e1);
    }
    ++prof->sweeps;
    ++prof->kernel_launches;
  }
  return DQ_OK;
}

int fused_run(double2* amp, uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_run_opts& o,
              FusedWork& fw, cudaStream_t st, int device, FusedHooks& hooks, dq_profile* prof,
              uint32_t* perm) {
  (void)device;
  Planner pl;
  pl.n = n;
  // thread geometry: DQSIM_SWEEP_TB=8 selects one 256-thread CTA per SM
  static const uint32_t tb_env = []() {
    const char* e = getenv("DQSIM_SWEEP_TB");
    return (e && atoi(e) == 8) ? 8u : 7u;
  }();
  const uint32_t TB = fw.plan_tb ? fw.plan_tb : tb_env;
  uint32_t M = TB + 4;  // 16 amplitudes per thread
  if (o.fusion_width >= (int)(TB + 2) && o.fusion_width <= (int)(TB + 4)) M = (uint32_t)o.fusion_width;
  if (M > n) M = n;
  pl.M = M;
  pl.TB = TB;
  pl.RB = M - TB;
  pl.single_tile = (M == n);
  // Pinned tile qubits: 0..4 (512-byte runs) or 0..2 (128-byte runs, two
  // more tile qubits free); by default each segment of 20+ qubits is planned
  // both ways and keeps the one with clearly fewer sweeps.
  // DQSIM_SWEEP_PIN=5 / 3 forces one.
  static const int pin_env = []() {
    const char* e = getenv("DQSIM_SWEEP_PIN");
    return e ? atoi(e) : 0;
  }();
  pl.pinned = pin_env == 3 ? 0x7ULL : 0x1FULL;
  pl.pin_auto = pin_env == 0 && n >= 20;
  if (o.max_cost > 0) pl.budget = (double)o.max_cost;
  Poly poly;
  poly.init(n);
  for (auto e : fw.events) cudaEventDestroy(e);
  fw.events.clear();
  const bool timing = o.time_sweeps != 0;

  // shots semantics: run the reference's fuse_circuit output
  std::vector<FusedEntry> fe;
  if (o.semantics == DQ_SEM_SHOTS) {
    fe = fuse_program(prog, ninst, n);
  } else {
    fe.resize(ninst);
    for (uint64_t i = 0; i < ninst; ++i) fe[i].inst = (int64_t)i;
  }

  std::vector<PGate> G;
  auto flush_segment = [&]() -> int {
    if (G.empty() && poly.empty()) return DQ_OK;
    int rc = fused_run_segment(amp, n, G, pl, poly, fw, st, timing, prof, hooks.lazy_basis);
    G.clear();
    return rc;
  };
  for (const FusedEntry& e : fe) {
    if (e.inst < 0) {  // a fused 2x2 of the shots path
      PGate g;
      const uint32_t t = perm[e.qubit];
      if (is_zero(e.m[1]) && is_zero(e.m[2]) && is_unit_phase(e.m[0]) && is_unit_phase(e.m[3])) {
        g.kind = PG_DIAG;
        if (!(e.m[0].re == 1.0 && e.m[0].im == 0.0)) g.cst = e.m[0];
        g.nlin = 1;
        g.lq[0] = t;
        g.lw[0] = (e.m[0].re == 1.0 && e.m[0].im == 0.0) ? e.m[3] : e.m[3] * conj(e.m[0]);
      } else {
        g.kind = PG_U1;
        g.t0 = t;
        for (int k = 0; k < 4; ++k) g.u[k] = e.m[k];
        g.real = e.m[0].im == 0.0 && e.m[1].im == 0.0 && e.m[2].im == 0.0 && e.m[3].im == 0.0;
      }
      g.touched = 1ULL << t;
      G.push_back(g);
      continue;
    }
    const dq_inst& in = prog[e.inst];
    const int64_t src = e.inst;
    // conditions are final: no measurement inside a segment
    bool ok = true;
    for (uint32_t c = 0; c < in.cond_count && ok; ++c) {
      const dq_cond& cd = hooks.conds[in.cond_first + c];
      uint64_t actual = 0;
      for (uint64_t b = 0; b < cd.creg_size; ++b) {
        const uint64_t idx = cd.creg_base + b;
        const uint64_t v = (idx < hooks.ncbits && hooks.cbits[idx] > 0) ? (uint64_t)hooks.cbits[idx] : 0;
        actual |= v << b;
      }
      ok = (actual == cd.creg_value);
    }
    if (!ok) continue;
    // While the state is still a pending basis vector and nothing has been
    // queued yet, an X gate is a flip of that basis index: exact, and it
    // leaves every tile qubit free for the gates that follow.
    if (in.kind == DQ_X && hooks.lazy_basis && *hooks.lazy_basis >= 0 && G.empty() &&
        poly.empty() && !poly.has_cst) {
      *hooks.lazy_basis ^= (int64_t)(1ULL << perm[in.q[0]]);
      continue;
    }
    switch (in.kind) {
      case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP:
        continue;
      case DQ_G_OPAQUE:
        if (o.semantics == DQ_SEM_SHOTS) continue;
        prof->failed_inst = src;
        return fail(DQ_ERR_UNSUPPORTED, "unsupported generic gate");
      case DQ_G_UNSUPPORTED:
        prof->failed_inst = src;
        return fail(DQ_ERR_UNSUPPORTED, "unsupported generic gate");
      case DQ_MEASURE:
      case DQ_RESET: {
        if (fw.plan_out) return fail(DQ_ERR_INVALID_ARG, "plan-only mode takes unitary programs");
        DQ_TRY(flush_segment());
        int out = 0;
        DQ_TRY(hooks.measure(perm[in.q[0]], &out));
        if (in.kind == DQ_MEASURE) {
          hooks.cbits[in.cbit] = out;
        } else if (out == 1) {
          GateOp op;
          hc xm[4] = {hc{0, 0}, hc{1, 0}, hc{1, 0}, hc{0, 0}};
          classify_1q(xm, perm[in.q[0]], 0, op);
          DQ_TRY(hooks.exact_gate(op));
        }
        continue;
      }
      default:
        break;
    }
    uint32_t sa = 0, sb = 0;
    bool is_swap = false;
    const size_t before = G.size();
    if (convert_inst(in, perm, G, &sa, &sb, &is_swap)) {
      if (is_swap) std::swap(perm[sa], perm[sb]);
      continue;
    }
    G.resize(before);
    if (fw.plan_out) return fail(DQ_ERR_INVALID_ARG, "plan-only mode: gate not representable");
    // not representable in a sweep: flush, then the exact per-gate kernel
    DQ_TRY(flush_segment());
    GateOp op;
    hc u[4];
    if (matrix_1q(in.kind, in.p, u)) {
      classify_1q(u, perm[in.q[0]], 0, op);
    } else {
      Gate g;
      if (!matrix_nq(in, g)) return fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
      for (uint32_t b = 0; b < g.k; ++b) g.qubits[b] = perm[g.qubits[b]];
      classify(g, op);
    }
    DQ_TRY(hooks.exact_gate(op));
  }
  DQ_TRY(flush_segment());
  if (timing && !fw.plan_out) {
    DQ_CUDA_TRY(cudaStreamSynchronize(st));
    double t = 0;
    for (size_t i = 0; i + 1 < fw.events.size(); i += 2) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, fw.events[i], fw.events[i + 1]);
      t += ms * 1e-3;
    }
    prof->sweep_time += t;
  }
  return DQ_OK;
}

int fused_plan(uint32_t n, const dq_inst* prog, uint64_t ninst, int semantics, uint32_t tb,
               int fusion_width, int64_t lazy_basis, std::vector<uint8_t>* blob,
               std::vector<uint64_t>* offs, uint32_t* perm, int64_t* synth, uint32_t* rb) {
  if (n < kFusedMinQubits || n > 34) return fail(DQ_ERR_INVALID_ARG, "fused planning needs 10..34 qubits");
  FusedWork fw;
  fw.plan_out = blob;
  fw.plan_offs = offs;
  fw.plan_tb = tb;
  FusedHooks hooks;
  int64_t lazy = lazy_basis;
  hooks.lazy_basis = lazy_basis >= 0 ? &lazy : nullptr;
  dq_profile prof{};
  prof.failed_inst = -1;
  dq_run_opts o{};
  o.semantics = semantics;
  o.exec = DQ_EXEC_FUSED;
  o.fusion_width = fusion_width;
  DQ_TRY(fused_run(nullptr, n, prog, ninst, o, fw, nullptr, 0, hooks, &prof, perm));
  *synth = offs->empty() ? (lazy_basis >= 0 ? lazy : -1) : fw.plan_synth;
  *rb = fw.plan_rb;
  return DQ_OK;
}

uint32_t sweep_run_bits(const uint8_t* prog) {
  return reinterpret_cast<const SwHeader*>(prog)->run_bits;
}

uint32_t sweep_prog_bytes(const uint8_t* prog) {
  return reinterpret_cast<const SwHeader*>(prog)->prog_bytes;
}

uint32_t sweep_flags(const uint8_t* prog) {
  return reinterpret_cast<const SwHeader*>(prog)->flags;
}

int launch_sweep_multi(const SweepJob* d_jobs, uint32_t njobs, uint32_t n, uint32_t rb,
                       uint32_t run_bits, uint32_t max_bytes, cudaStream_t st, uint32_t flags) {
  if (!njobs) return DQ_OK;
  if (n < 7 + rb) return fail(DQ_ERR_INVALID_ARG, "state smaller than a tile");
  if (max_bytes > (uint32_t)max_prog(7 + (int)rb)) return fail(DQ_ERR_INTERNAL, "sweep program too large");
  const bool r3 = run_bits == 3;
  switch (rb) {
    case 2: return r3 ? launch_sweep_multi_t<7, 2, 3>(d_jobs, njobs, n, max_bytes, st)
                      : launch_sweep_multi_t<7, 2, 5>(d_jobs, njobs, n, max_bytes, st);
    case 3: return r3 ? launch_sweep_multi_t<7, 3, 3>(d_jobs, njobs, n, max_bytes, st)
                      : launch_sweep_multi_t<7, 3, 5>(d_jobs, njobs, n, max_bytes, st);
    case 4:
      // every job's program allows a restricted build (the flags of all of them ANDed)
      if (flags & SWF_HONLY)
        return r3 ? launch_sweep_multi_t<7, 4, 3, FORM_H>(d_jobs, njobs, n, max_bytes, st)
                  : launch_sweep_multi_t<7, 4, 5, FORM_H>(d_jobs, njobs, n, max_bytes, st);
      if (flags & SWF_RONLY)
        return r3 ? launch_sweep_multi_t<7, 4, 3, FORM_R>(d_jobs, njobs, n, max_bytes, st)
                  : launch_sweep_multi_t<7, 4, 5, FORM_R>(d_jobs, njobs, n, max_bytes, st);
      if (flags & SWF_UONLY)
        return r3 ? launch_sweep_multi_t<7, 4, 3, FORM_U>(d_jobs, njobs, n, max_bytes, st)
                  : launch_sweep_multi_t<7, 4, 5, FORM_U>(d_jobs, njobs, n, max_bytes, st);
      return r3 ? launch_sweep_multi_t<7, 4, 3>(d_jobs, njobs, n, max_bytes, st)
                : launch_sweep_multi_t<7, 4, 5>(d_jobs, njobs, n, max_bytes, st);
    default: return fail(DQ_ERR_INTERNAL, "unsupported multi-sweep geometry");
  }
}

}  // namespace dq
