// dq_traj.cu — batched shot trajectories in one persistent launch.
//
// simulate_shots (statevector/simulator.rs:216-322) runs every shot as its
// own trajectory: a fresh |0..0> state, the fused program (types.rs:248-293,
// run_fused_par 870-884, run_instruction_par 638-864), mid-circuit measure /
// reset / conditionals, and ChaCha8Rng::seed_from_u64(base_seed + i).  Here
// each trajectory lives entirely in shared memory: a thread-block cluster of
// 2^cb CTAs holds one 2^n-amplitude state (2^(n-cb) amplitudes per CTA, at
// most 8192 = 128 KiB), so n <= 16 with clusters of up to 8 CTAs.  Gates on
// the low n-cb qubits touch one CTA's shared memory; gates on the top cb
// qubits pair elements across CTAs through distributed shared memory.  A
// measurement reduces p1 per CTA (fixed order), exchanges the cluster's
// partials, draws the outcome from the device ChaCha8 stream and collapses
// in place.  Each cluster loops over trajectories until all shots are done;
// the state never touches HBM, only the classical registers are written out.
//
// Arithmetic is the exact per-gate arithmetic of dq_engine.cu (num-complex
// order, no FMA, zero matrix entries skipped), so amplitudes match the
// oracle's sequential shot bit for bit; p1 is summed in a different order,
// which can only change an outcome when the draw lies within rounding of
// p1 — such draws (|r - p1| < 1e-12) are counted and reported.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "dq_common.cuh"
#include "dq_fused.cuh"
#include "dq_gates.hpp"
#include "dq_handle.cuh"
#include "dq_rng.cuh"
#include "dq_sweep.cuh"

namespace cg = cooperative_groups;

namespace dq {
namespace {

constexpr uint32_t kLocalBitsMax = 13;  // 8192 amplitudes = 128 KiB per CTA
// Tile bits of the fused sweeps that HBM-resident batch items run (2^12
// amplitudes: 8 thread bits of the 256-thread CTA and 4 register bits).
constexpr int kHbmTileBits = 12;
constexpr uint32_t kTrajMaxQubits = 16;
constexpr uint32_t kTrajMaxCbits = 1024;

enum TOpType : uint8_t {
  T_NOP = 0, T_ONEQ, T_PHASE, T_XPERM, T_SWAP, T_DIAG, T_DENSE, T_MEASURE, T_RESET, T_FAIL,
  T_RPHASE  // header of k (>= 2) T_ONEQ / T_XPERM ops on the four local bits q[0..3]
};

struct TOp {
  uint8_t type;
  uint8_t k;        // DIAG / DENSE: qubit count
  uint8_t t1, t2;   // target(s)
  uint32_t cond_first, cond_count;
  int32_t cbit;     // MEASURE: classical bit; FAIL: unused
  uint32_t mat;     // offset into the matrix pool (double2 units)
  uint32_t remote;  // touches cluster qubits or needs a cluster reduction
  uint64_t ctrl;    // control mask (all must be 1)
  uint8_t q[8];     // DIAG / DENSE qubits, q[0] = MSB of the matrix index; RPHASE: register bits
  int64_t inst;     // original instruction index (-1: a fused 2x2)
};
static_assert(sizeof(TOp) == 48, "TOp layout");

struct TProg {         // one program of a launch
  uint32_t ops_off, nops;
  uint32_t n, lb;       // qubits; amplitudes per CTA = 2^lb
  uint32_t ncbits, pad;
  uint64_t base_seed;   // shot s draws from seed_from_u64(base_seed + s) (wrapping)
  uint64_t cbits_off;   // shot s writes cbits_out[cbits_off + s * ncbits ...]
  double2* state_out;   // device: final state of shot s at + s * 2^n, or null
  // Items too large for a cluster's shared memory (batch items of 17+ qubits)
  // keep their state in HBM at `hbm` and run as fused tile sweeps: sweeps
  // [sweep_first, sweep_first + nsweeps) of the launch's sweep table, the
  // first one generating its tiles from the basis index `synth`.
  double2* hbm;
  uint32_t sweep_first, nsweeps;
  long long synth;
};
struct TSweep {          // one fused sweep of an HBM item
  uint64_t off;          // byte offset of its program in the launch's sweep blob
  uint32_t ntiles, run_bits;
  uint32_t prog_bytes, pad;
};
struct TItem {          // one trajectory: a shot of a program
  uint32_t prog, pad;
  uint64_t shot;
};
struct TrajParams {
  const TOp* ops;
  const double2* pool;
  const dq_cond* conds;
  const TProg* progs;
  const TItem* items;
  int32_t* cbits_out;
  unsigned long long* queue;     // work queue: next item index
  unsigned long long* boundary;  // draws within 1e-12 of p1
  long long* failed;             // lowest (prog << 40 | instruction) that failed
  uint64_t nitems;
  const uint8_t* sweep_blob;     // sweep programs of the HBM items (dq_sweep.cuh layout)
  const TSweep* sweeps;
};

__device__ __forceinline__ uint32_t ins0(uint32_t k, uint32_t p) {
  return ((k >> p) << (p + 1)) | (k & ((1u << p) - 1u));
}

// Shared-memory layout of a trajectory slice: logical element o lives at
// tswz(o).  The low three index bits are XORed with a fold of the higher ones
// so that eight threads touching elements that differ only in higher bits
// (pairs of a low target, strided controls) use eight different bank rows.
// The same bijection in every CTA keeps distributed-shared-memory accesses
// consistent; summation orders follow logical indices, so results are
// unchanged.
__device__ __forceinline__ uint32_t tswz(uint32_t o) {
  return o ^ (((o >> 3) ^ (o >> 6) ^ (o >> 9) ^ (o >> 12)) & 7u);
}

// One op of a register phase on the 16 amplitudes a thread holds (register
// index bit b = local qubit q[b] of the phase): the exact per-pair arithmetic
// of the shared-memory path, for the pairs whose control bits (creg) are set.
template <int RT>
__device__ __forceinline__ void rphase_1q(double2 (&a)[16], const double2 (&u)[4], uint32_t creg) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << RT)) continue;
    if (((uint32_t)j & creg) != creg) continue;
    const int k = j | (1 << RT);
    const double2 x = a[j], y = a[k];
    a[j] = cadd_x(cmul_x(u[0], x), cmul_x(u[1], y));
    a[k] = cadd_x(cmul_x(u[2], x), cmul_x(u[3], y));
  }
}
template <int RT>
__device__ __forceinline__ void rphase_x(double2 (&a)[16], uint32_t creg) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << RT)) continue;
    if (((uint32_t)j & creg) != creg) continue;
    const int k = j | (1 << RT);
    const double2 x = a[j];
    a[j] = a[k];
    a[k] = x;
  }
}

// Fixed-order block sum, result broadcast to every thread.
template <int THREADS>
__device__ double block_sum_all(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int i = 0; i < THREADS / 32; ++i) a = __dadd_rn(a, sh[i]);
    sh[32] = a;
  }
  __syncthreads();
  return sh[32];
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_traj(const TrajParams P) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double s_bcast[2];
  __shared__ int s_skip[2];  // double-buffered by op parity: one barrier per op suffices
  __shared__ unsigned long long s_item;

  cg::cluster_group cl = cg::this_cluster();
  const uint32_t C = cl.num_blocks(), rank = cl.block_rank();
  const uint32_t tid = threadIdx.x;
  auto sync_all = [&](bool cluster) {
    if (cluster && C > 1) cl.sync(); else __syncthreads();
  };

  for (;;) {
    // rank 0 takes the next trajectory from the queue and shares it
    if (rank == 0 && tid == 0) s_item = atomicAdd(P.queue, 1ULL);
    sync_all(true);
    const unsigned long long item = (rank == 0) ? s_item : *cl.map_shared_rank(&s_item, 0);
    if (item >= P.nitems) {
      sync_all(true);  // no CTA leaves while another still reads its shared memory
      break;
    }
    const TItem it = P.items[item];
    const TProg pg = P.progs[it.prog];
    if (pg.hbm) {
      // HBM item: the cluster's CTAs split the tiles of each sweep (tiles
      // rank, rank + C, ...; 256 threads run the 8-thread-bit geometry the
      // sweeps were planned for) with a cluster barrier between sweeps; the
      // fence makes each sweep's stores visible to the CTAs of the next one.
      // Each sweep's program is staged in shared memory behind two tile
      // buffers (the next tile loads while the current one is computed).
      if constexpr (THREADS == 256) {
        double2* bufs = reinterpret_cast<double2*>(smraw);
        double2* slots = bufs + 2 * (1u << kHbmTileBits);
        uint8_t* sprog = reinterpret_cast<uint8_t*>(slots + kMaxSlots);
        if (pg.nsweeps == 0) {  // nothing but a basis state to write
          const uint64_t len = 1ULL << pg.n;
          for (uint64_t i = (uint64_t)rank * THREADS + tid; i < len; i += (uint64_t)C * THREADS)
            pg.hbm[i] = make_double2(i == (uint64_t)pg.synth ? 1.0 : 0.0, 0.0);
        }
        for (uint32_t s = 0; s < pg.nsweeps; ++s) {
          const TSweep sw = P.sweeps[pg.sweep_first + s];
          const long long sy = s == 0 ? pg.synth : -1LL;
          for (uint32_t i = tid * 16u; i < sw.prog_bytes; i += THREADS * 16u)
            *reinterpret_cast<uint4*>(sprog + i) =
                __ldg(reinterpret_cast<const uint4*>(P.sweep_blob + sw.off + i));
          __syncthreads();
          if (sw.run_bits == 3)
            sweep_tiles<8, kHbmTileBits - 8, 2, 3>(pg.hbm, sprog, sw.ntiles, sy, bufs, slots, rank, C);
          else
            sweep_tiles<8, kHbmTileBits - 8, 2, 5>(pg.hbm, sprog, sw.ntiles, sy, bufs, slots, rank, C);
          __threadfence();
          cl.sync();
        }
      }
      if (rank == 0)  // unitary items write no classical bit
        for (uint32_t i = tid; i < pg.ncbits; i += THREADS)
          P.cbits_out[pg.cbits_off + it.shot * pg.ncbits + i] = -1;
      sync_all(true);
      continue;
    }
    const uint32_t lb = pg.lb, L = 1u << lb;
    double2* sm = reinterpret_cast<double2*>(smraw);
    double* red = reinterpret_cast<double*>(sm + L);    // [0..32]: block sums, [40]: CTA partial
    int32_t* cb = reinterpret_cast<int32_t*>(red + 48);  // classical bits
    const uint64_t gbase = (uint64_t)rank << lb;
    const uint64_t lmask = (uint64_t)L - 1;
    auto elem = [&](uint64_t g) -> double2* {
      const uint32_t r = (uint32_t)(g >> lb);
      double2* base = (r == rank) ? sm : cl.map_shared_rank(sm, r);
      return base + tswz((uint32_t)(g & lmask));
    };

    uint32_t key[8];
    seed_key_from_u64(pg.base_seed + it.shot, key);
    uint64_t draws = 0;
    for (uint32_t i = tid; i < L; i += THREADS) sm[i] = make_double2(0.0, 0.0);
    for (uint32_t i = tid; i < pg.ncbits; i += THREADS) cb[i] = -1;
    if (rank == 0 && tid == 0) sm[0] = make_double2(1.0, 0.0);
    bool last_cluster = true;
    sync_all(true);

    // the next op's descriptor and one-qubit matrix are loaded while the
    // current op runs (global loads, otherwise a round trip before every op)
    TOp nxt{};
    double2 nu[4] = {};
    auto fetch = [&](uint32_t k) {
      nxt = P.ops[pg.ops_off + k];
      if (nxt.type == T_ONEQ)
        for (int i = 0; i < 4; ++i) nu[i] = P.pool[nxt.mat + i];
    };
    if (pg.nops) fetch(0);
    for (uint32_t oi = 0; oi < pg.nops; ++oi) {
      const TOp op = nxt;
      double2 u[4];
      for (int i = 0; i < 4; ++i) u[i] = nu[i];
      if (oi + 1 < pg.nops) fetch(oi + 1);
      // conditions (little-endian register value, unwritten bits read as 0)
      if (op.cond_count) {
        if (tid == 0) {
          int ok = 1;
          for (uint32_t c = 0; c < op.cond_count && ok; ++c) {
            const dq_cond cd = P.conds[op.cond_first + c];
            uint64_t actual = 0;
            for (uint64_t b = 0; b < cd.creg_size; ++b) {
              const uint64_t idx = cd.creg_base + b;
              const int32_t v = (idx < pg.ncbits) ? cb[idx] : 0;
              actual |= (uint64_t)(v > 0 ? v : 0) << b;
            }
            if (actual != cd.creg_value) ok = 0;
          }
          s_skip[oi & 1] = !ok;
        }
        __syncthreads();
        if (s_skip[oi & 1]) continue;
      }
      const bool remote = op.remote && C > 1;
      if (remote && !last_cluster) cl.sync();

      switch (op.type) {
        case T_ONEQ:
        case T_XPERM: {
          const uint32_t t = op.t1;
          const uint64_t hi_ctrl = op.ctrl & ~lmask;
          const uint32_t lo_ctrl = (uint32_t)(op.ctrl & lmask);
          // local zero-insertion positions: target (if local) and local controls
          // local zero-insertion positions (the set bits of zmask, ascending;
          // no array: a dynamically indexed one would live in local memory)
          const uint64_t zmask = lo_ctrl | (t < lb ? (1ULL << t) : 0ULL);
          const int np = __popcll((long long)zmask);
          const uint32_t count = L >> np;
          const uint32_t p0 = np > 0 ? (uint32_t)(__ffsll((long long)zmask) - 1) : 0u;
          const uint64_t zm1 = zmask & (zmask - 1);
          const uint32_t p1 = np > 1 ? (uint32_t)(__ffsll((long long)zm1) - 1) : 0u;
          // pair k -> swizzled index of its element with the target bit 0
          auto index = [&](uint32_t k) -> uint32_t {
            uint32_t o;
            if (np == 1) {
              o = ins0(k, p0);
            } else if (np == 2) {
              o = ins0(ins0(k, p0), p1);
            } else {
              o = k;
              for (uint64_t mm = zmask; mm; mm &= mm - 1) o = ins0(o, (uint32_t)(__ffsll((long long)mm) - 1));
            }
            return tswz(o | lo_ctrl);
          };
          double2 *A, *B;
          uint32_t sx, lo, hi;
          if (t < lb) {
            if ((gbase & hi_ctrl) != hi_ctrl) break;
            A = B = sm;
            sx = tswz(1u << t);  // tswz is linear over XOR: partner = index ^ tswz(target bit)
            lo = 0;
            hi = count;
          } else {
            const uint32_t tbr = 1u << (t - lb);
            const uint32_t r0 = rank & ~tbr, r1 = rank | tbr;
            if ((((uint64_t)r0 << lb) & hi_ctrl) != hi_ctrl) break;
            A = (r0 == rank) ? sm : cl.map_shared_rank(sm, r0);
            B = (r1 == rank) ? sm : cl.map_shared_rank(sm, r1);
            sx = 0;
            const uint32_t half = count > 1 ? count >> 1 : 1;
            if (rank == r0) { lo = 0; hi = half; } else { lo = half; hi = count > 1 ? count : half; }
          }
          // four pairs per thread in flight: loads first, then the exact
          // per-pair arithmetic (pairs are disjoint, so the order of the
          // stores does not matter)
          for (uint32_t k0 = lo + tid; k0 < hi; k0 += 4u * THREADS) {
            uint32_t so[4];
            double2 a[4], b[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              const uint32_t k = k0 + (uint32_t)v * THREADS;
              so[v] = index(k < hi ? k : k0);
              a[v] = A[so[v]];
              b[v] = B[so[v] ^ sx];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              if (k0 + (uint32_t)v * THREADS >= hi) break;
              if (op.type == T_ONEQ) {
                A[so[v]] = cadd_x(cmul_x(u[0], a[v]), cmul_x(u[1], b[v]));
                B[so[v] ^ sx] = cadd_x(cmul_x(u[2], a[v]), cmul_x(u[3], b[v]));
              } else {
                A[so[v]] = b[v];
                B[so[v] ^ sx] = a[v];
              }
            }
          }
          break;
        }
        case T_PHASE: {
          const uint64_t need = op.ctrl | (1ULL << op.t1);
          const uint64_t hi = need & ~lmask, lo = need & lmask;
          if ((gbase & hi) != hi) break;
          const double2 e = P.pool[op.mat];
          const int np = __popcll((long long)lo);
          const uint32_t count = L >> np;
          const uint32_t p0 = np > 0 ? (uint32_t)(__ffsll((long long)lo) - 1) : 0u;
          const uint64_t lo1 = lo & (lo - 1);
          const uint32_t p1 = np > 1 ? (uint32_t)(__ffsll((long long)lo1) - 1) : 0u;
          for (uint32_t k0 = tid; k0 < count; k0 += 4u * THREADS) {
            uint32_t so[4];
            double2 a[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              const uint32_t k = k0 + (uint32_t)v * THREADS < count ? k0 + (uint32_t)v * THREADS : k0;
              uint32_t o;
              if (np == 1) {
                o = ins0(k, p0);
              } else if (np == 2) {
                o = ins0(ins0(k, p0), p1);
              } else {
                o = k;
                for (uint64_t mm = lo; mm; mm &= mm - 1) o = ins0(o, (uint32_t)(__ffsll((long long)mm) - 1));
              }
              so[v] = tswz(o | (uint32_t)lo);
              a[v] = sm[so[v]];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              if (k0 + (uint32_t)v * THREADS >= count) break;
              sm[so[v]] = cmul_x(e, a[v]);
            }
          }
          break;
        }
        case T_DIAG: {
          const uint32_t kq = op.k;
          for (uint32_t o = tid; o < L; o += THREADS) {
            const uint64_t g = gbase | o;
            uint32_t idx = 0;
            for (uint32_t b = 0; b < kq; ++b) idx = (idx << 1) | (uint32_t)((g >> op.q[b]) & 1ULL);
            const double2 d = P.pool[op.mat + idx];
            if (d.x == 1.0 && d.y == 0.0) continue;
            sm[tswz(o)] = cmul_x(d, sm[tswz(o)]);
          }
          break;
        }
        case T_SWAP: {
          // pairs (i: t1 = 1, t2 = 0) <-> (j = i ^ both); the CTA owning i does the pair
          const uint64_t b1 = 1ULL << op.t1, b2 = 1ULL << op.t2;
          const uint64_t fixed1 = op.ctrl | b1;  // bits that must be 1 in i
          const uint64_t gate = op.ctrl | b1 | b2;
          const uint64_t hi_one = fixed1 & ~lmask, hi_zero = b2 & ~lmask;
          if ((gbase & hi_one) != hi_one || (gbase & hi_zero) != 0) break;
          const uint64_t zmask = gate & lmask;
          const uint32_t count = L >> __popcll((long long)zmask);
          const uint32_t lo_one = (uint32_t)(fixed1 & lmask);
          for (uint32_t k = tid; k < count; k += THREADS) {
            uint32_t o = k;
            for (uint64_t mm = zmask; mm; mm &= mm - 1) o = ins0(o, (uint32_t)(__ffsll((long long)mm) - 1));
            o |= lo_one;
            const uint64_t gi = gbase | o, gj = gi ^ b1 ^ b2;
            double2* pi = sm + tswz(o);
            double2* pj = elem(gj);
            const double2 a = *pi, b = *pj;
            *pi = b;
            *pj = a;
          }
          break;
        }
        case T_DENSE: {
          const uint32_t kq = op.k, D = 1u << kq;
          uint64_t gm = 0;
          for (uint32_t b = 0; b < kq; ++b) gm |= 1ULL << op.q[b];
          if ((gbase & gm & ~lmask) != 0) break;  // group base must have the gate bits zero
          const uint64_t zmask = gm & lmask;
          const uint32_t count = L >> __popcll((long long)zmask);
          for (uint32_t k = tid; k < count; k += THREADS) {
            uint32_t o = k;
            for (uint64_t mm = zmask; mm; mm &= mm - 1) o = ins0(o, (uint32_t)(__ffsll((long long)mm) - 1));
            const uint64_t base = gbase | o;
            double2 v[32];
            double2* ptr[32];
            for (uint32_t j = 0; j < D; ++j) {
              uint64_t off = 0;
              for (uint32_t b = 0; b < kq; ++b)
                if ((j >> (kq - 1 - b)) & 1u) off |= 1ULL << op.q[b];
              ptr[j] = elem(base | off);
              v[j] = *ptr[j];
            }
            for (uint32_t r = 0; r < D; ++r) {
              double2 acc = make_double2(0.0, 0.0);
              for (uint32_t c = 0; c < D; ++c) {
                const double2 uu = P.pool[op.mat + r * D + c];
                if (uu.x != 0.0 || uu.y != 0.0) acc = cadd_x(acc, cmul_x(uu, v[c]));
              }
              *ptr[r] = acc;
            }
          }
          break;
        }
        case T_MEASURE:
        case T_RESET: {
          const uint32_t q = op.t1;
          const uint64_t qb = 1ULL << q;
          double part = 0.0;
          if (q < lb) {
            for (uint32_t k = tid; k < L / 2; k += THREADS)
              part = __dadd_rn(part, norm_sqr_x(sm[tswz(ins0(k, q) | (uint32_t)qb)]));
          } else if (gbase & qb) {
            for (uint32_t o = tid; o < L; o += THREADS) part = __dadd_rn(part, norm_sqr_x(sm[tswz(o)]));
          }
          const double cta = block_sum_all<THREADS>(part, red);
          if (tid == 0) red[40] = cta;
          if (C > 1) cl.sync(); else __syncthreads();
          if (tid == 0) {
            double p1 = 0.0;
            for (uint32_t r = 0; r < C; ++r) {
              const double* pr = (r == rank) ? red : cl.map_shared_rank(red, r);
              p1 = __dadd_rn(p1, pr[40]);
            }
            const double rr = chacha8_draw(key, draws);
            const int o = rr < p1 ? 1 : 0;
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
            if (rank == 0 && fabs(rr - p1) < 1e-12) atomicAdd(P.boundary, 1ULL);
            s_bcast[0] = (double)o;
            s_bcast[1] = norm;
            if (op.type == T_MEASURE) cb[op.cbit] = o;
          }
          ++draws;
          __syncthreads();
          const int o = (int)s_bcast[0];
          const double norm = s_bcast[1];
          for (uint32_t i = tid; i < L; i += THREADS) {
            const bool set = ((gbase | i) & qb) != 0;
            if (set != (o == 1)) {
              sm[tswz(i)] = make_double2(0.0, 0.0);
            } else {
              const double2 a = sm[tswz(i)];
              sm[tswz(i)] = make_double2(__ddiv_rn(a.x, norm), __ddiv_rn(a.y, norm));
            }
          }
          if (op.type == T_RESET && o == 1) {
            // X on q: an exact exchange of the two halves
            if (C > 1) cl.sync(); else __syncthreads();
            if (q < lb) {
              for (uint32_t k = tid; k < L / 2; k += THREADS) {
                const uint32_t a0 = ins0(k, q), a1 = a0 | (uint32_t)qb;
                const double2 x = sm[tswz(a0)];
                sm[tswz(a0)] = sm[tswz(a1)];
                sm[tswz(a1)] = x;
              }
            } else {
              const uint32_t tbr = 1u << (q - lb);
              if (!(rank & tbr)) {
                double2* other = cl.map_shared_rank(sm, rank | tbr);
                for (uint32_t i = tid; i < L; i += THREADS) {
                  const double2 x = sm[i];
                  sm[i] = other[i];
                  other[i] = x;
                }
              }
            }
          }
          break;
        }
        case T_RPHASE: {
          // the next op.k ops act on the four local bits q[0..3] only: each
          // thread holds the 16 amplitudes of a group in registers and applies
          // them in program order (one shared-memory pass, one barrier)
          const uint32_t cnt = op.k;
          const uint32_t r0 = op.q[0], r1 = op.q[1], r2 = op.q[2], r3 = op.q[3];
          const uint32_t s0 = tswz(1u << r0), s1 = tswz(1u << r1), s2 = tswz(1u << r2),
                         s3 = tswz(1u << r3);
          auto sidx = [&](uint32_t sb, int j) {
            return sb ^ ((j & 1) ? s0 : 0u) ^ ((j & 2) ? s1 : 0u) ^ ((j & 4) ? s2 : 0u) ^
                   ((j & 8) ? s3 : 0u);
          };
          const uint32_t groups = L >> 4;
          for (uint32_t gi = tid; gi < groups; gi += THREADS) {
            // tswz is linear over XOR and the group base has the register bits clear
            const uint32_t sb = tswz(ins0(ins0(ins0(ins0(gi, r0), r1), r2), r3));
            double2 a[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = sm[sidx(sb, j)];
            for (uint32_t sidx_op = 0; sidx_op < cnt; ++sidx_op) {
              const TOp so = P.ops[pg.ops_off + oi + 1 + sidx_op];
              const uint32_t t = so.t1;
              const uint32_t rt = t == r0 ? 0u : (t == r1 ? 1u : (t == r2 ? 2u : 3u));
              uint32_t creg = 0;
              if (so.ctrl) {
                if ((so.ctrl >> r0) & 1ULL) creg |= 1u;
                if ((so.ctrl >> r1) & 1ULL) creg |= 2u;
                if ((so.ctrl >> r2) & 1ULL) creg |= 4u;
                if ((so.ctrl >> r3) & 1ULL) creg |= 8u;
              }
              if (so.type == T_ONEQ) {
                double2 uu[4];
                for (int i = 0; i < 4; ++i) uu[i] = P.pool[so.mat + i];
                switch (rt) {
                  case 0: rphase_1q<0>(a, uu, creg); break;
                  case 1: rphase_1q<1>(a, uu, creg); break;
                  case 2: rphase_1q<2>(a, uu, creg); break;
                  default: rphase_1q<3>(a, uu, creg); break;
                }
              } else {
                switch (rt) {
                  case 0: rphase_x<0>(a, creg); break;
                  case 1: rphase_x<1>(a, creg); break;
                  case 2: rphase_x<2>(a, creg); break;
                  default: rphase_x<3>(a, creg); break;
                }
              }
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) sm[sidx(sb, j)] = a[j];
          }
          // continue after the phase's ops
          oi += cnt;
          if (oi + 1 < pg.nops) fetch(oi + 1);
          break;
        }
        case T_FAIL:
          if (tid == 0 && rank == 0) atomicMin(P.failed, ((long long)it.prog << 40) | op.inst);
          break;
        default:
          break;
      }
      sync_all(remote);
      last_cluster = remote || C == 1;
      if (op.type == T_FAIL) break;
    }
    // classical bits and (optionally) the final state out; the next
    // trajectory re-initialises after a cluster barrier
    if (rank == 0)
      for (uint32_t i = tid; i < pg.ncbits; i += THREADS)
        P.cbits_out[pg.cbits_off + it.shot * pg.ncbits + i] = cb[i];
    if (pg.state_out) {
      double2* dst = pg.state_out + (it.shot << pg.n) + gbase;
      for (uint32_t i = tid; i < L; i += THREADS) dst[i] = sm[tswz(i)];
    }
    sync_all(true);
  }
}

// ---- host side ---------------------------------------------------------------

struct Encoded {
  std::vector<TOp> ops;
  std::vector<double2> pool;
};

uint32_t push_mat(Encoded& e, const hc* m, uint32_t count) {
  const uint32_t off = (uint32_t)e.pool.size();
  for (uint32_t i = 0; i < count; ++i) e.pool.push_back(make_double2(m[i].re, m[i].im));
  return off;
}

TOp blank_op(int64_t inst, const dq_inst* in) {
  TOp t{};
  t.inst = inst;
  t.cbit = -1;
  if (in) {
    t.cond_first = in->cond_first;
    t.cond_count = in->cond_count;
  }
  return t;
}

void encode_gateop(Encoded& e, const GateOp& g, TOp t) {
  switch (g.cls) {
    case GC_ONE_Q:
      t.type = T_ONEQ;
      t.t1 = (uint8_t)g.target;
      t.ctrl = g.ctrl_mask;
      t.mat = push_mat(e, g.u, 4);
      break;
    case GC_PHASE:
      t.type = T_PHASE;
      t.t1 = (uint8_t)g.target;
      t.ctrl = g.ctrl_mask;
      t.mat = push_mat(e, g.u, 1);
      break;
    case GC_XPERM:
      t.type = T_XPERM;
      t.t1 = (uint8_t)g.target;
      t.ctrl = g.ctrl_mask;
      break;
    case GC_SWAP:
      t.type = T_SWAP;
      t.t1 = (uint8_t)g.target;
      t.t2 = (uint8_t)g.target2;
      t.ctrl = g.ctrl_mask;
      break;
    case GC_DIAG: {
      t.type = T_DIAG;
      t.k = (uint8_t)g.dense.k;
      for (uint32_t b = 0; b < g.dense.k; ++b) t.q[b] = (uint8_t)g.dense.qubits[b];
      const uint32_t D = 1u << g.dense.k;
      std::vector<hc> d(D);
      for (uint32_t i = 0; i < D; ++i) d[i] = g.dense.m[i * D + i];
      t.mat = push_mat(e, d.data(), D);
      break;
    }
    case GC_DENSE: {
      t.type = T_DENSE;
      t.k = (uint8_t)g.dense.k;
      for (uint32_t b = 0; b < g.dense.k; ++b) t.q[b] = (uint8_t)g.dense.qubits[b];
      const uint32_t D = 1u << g.dense.k;
      t.mat = push_mat(e, g.dense.m, D * D);
      break;
    }
    default:
      t.type = T_NOP;
      break;
  }
  e.ops.push_back(t);
}

// The fused shot program (fuse_program) as device ops, appended to e.
int encode_program(const dq_inst* prog, uint64_t ninst, uint32_t n, uint32_t cond_base,
                   Encoded& e) {
  const std::vector<FusedEntry> fused = fuse_program(prog, ninst, n);
  for (const FusedEntry& f : fused) {
    if (f.inst < 0) {
      GateOp g;
      classify_1q(f.m, f.qubit, 0, g);
      encode_gateop(e, g, blank_op(-1, nullptr));
      continue;
    }
    const dq_inst& in = prog[f.inst];
    TOp t = blank_op(f.inst, &in);
    t.cond_first += cond_base;
    switch (in.kind) {
      case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP:
      case DQ_G_OPAQUE:  // a no-op in the shot path (run_instruction_par)
        continue;
      case DQ_G_UNSUPPORTED:
        t.type = T_FAIL;
        e.ops.push_back(t);
        continue;
      case DQ_MEASURE:
        t.type = T_MEASURE;
        t.t1 = (uint8_t)in.q[0];
        t.cbit = (int32_t)in.cbit;
        e.ops.push_back(t);
        continue;
      case DQ_RESET:
        t.type = T_RESET;
        t.t1 = (uint8_t)in.q[0];
        e.ops.push_back(t);
        continue;
      default:
        break;
    }
    GateOp g;
    if (!inst_to_op(in, g)) return fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
    encode_gateop(e, g, t);
  }
  return DQ_OK;
}

void mark_remote(TOp* ops, size_t count, uint32_t lb) {
  const uint64_t lmask = (1ULL << lb) - 1;
  for (size_t i = 0; i < count; ++i) {
    TOp& t = ops[i];
    uint64_t touched = 0;
    switch (t.type) {
      case T_ONEQ: case T_XPERM: touched = 1ULL << t.t1; break;
      case T_SWAP: touched = (1ULL << t.t1) | (1ULL << t.t2); break;
      case T_DENSE:
        for (uint32_t b = 0; b < t.k; ++b) touched |= 1ULL << t.q[b];
        break;
      case T_MEASURE: case T_RESET: t.remote = 1; continue;
      default: break;
    }
    t.remote = (touched & ~lmask) ? 1u : 0u;
  }
}

// Register phases: maximal runs (two or more) of unconditional T_ONEQ /
// T_XPERM ops whose targets and controls all lie within four local bits
// become one T_RPHASE header followed by the ops (in program order).
std::vector<TOp> group_phases(const std::vector<TOp>& ops, uint32_t lb) {
  std::vector<TOp> out;
  if (lb < 4) return ops;
  const uint64_t lmask = (1ULL << lb) - 1;
  auto bits_of = [](const TOp& t) { return t.ctrl | (1ULL << t.t1); };
  auto eligible = [&](const TOp& t) {
    return (t.type == T_ONEQ || t.type == T_XPERM) && t.cond_count == 0 && !t.remote &&
           (bits_of(t) & ~lmask) == 0;
  };
  size_t i = 0;
  while (i < ops.size()) {
    if (!eligible(ops[i])) {
      out.push_back(ops[i++]);
      continue;
    }
    uint64_t set = bits_of(ops[i]);
    size_t j = i + 1;
    while (j < ops.size() && j - i < 255 && eligible(ops[j]) &&
           __builtin_popcountll(set | bits_of(ops[j])) <= 4) {
      set |= bits_of(ops[j]);
      ++j;
    }
    if (j - i < 2 || __builtin_popcountll(set) > 4) {
      out.push_back(ops[i++]);
      continue;
    }
    for (uint32_t b = 0; b < lb && __builtin_popcountll(set) < 4; ++b) set |= 1ULL << b;
    TOp h{};
    h.type = T_RPHASE;
    h.k = (uint8_t)(j - i);
    h.inst = ops[i].inst;
    int nb = 0;
    for (uint32_t b = 0; b < lb; ++b)
      if ((set >> b) & 1ULL) h.q[nb++] = (uint8_t)b;
    out.push_back(h);
    for (size_t k = i; k < j; ++k) out.push_back(ops[k]);
    i = j;
  }
  return out;
}

// All programs and trajectories of one launch (one cluster span).
struct LaunchSet {
  Encoded enc;
  std::vector<dq_cond> conds;
  std::vector<TProg> progs;
  std::vector<TItem> items;
  std::vector<uint8_t> blob;     // sweep programs of the HBM items
  // or, when set, the sweep programs staged in pinned host memory
  const uint8_t* blob_host = nullptr;
  size_t blob_host_bytes = 0;
  std::vector<TSweep> sweeps;
  uint32_t C = 1;
  uint32_t max_lb = 1, max_ncbits = 0;
  size_t hbm_smem = 0;           // shared memory the HBM items' sweeps need
};

// Largest batch item that runs as HBM-resident fused sweeps inside the
// persistent launch (2^30 amplitudes = 16 GiB).
constexpr uint32_t kHbmItemMaxQubits = 30;
// Sweep geometry of HBM items: 8 thread bits (the 256-thread trajectory
// CTA), 4 register bits, tiles of 2^12 amplitudes (two tile buffers, the
// slot factors and the staged program fit one CTA's shared memory).
constexpr uint32_t kHbmTB = 8, kHbmM = kHbmTileBits;

// A unitary batch item planned as fused sweeps for the HBM path of k_traj.
struct HbmPlan {
  std::vector<uint8_t> blob;
  std::vector<uint64_t> offs;
  int64_t synth = -1;
  uint32_t perm[64];
};

// Plans item `it` (shot semantics, from |0...0>) as sweeps of the HBM
// geometry; false when the item has measurements, resets or conditions, or a
// gate the sweep planner does not represent (such items run on the engine).
bool plan_hbm_item(const dq_batch_item& it, HbmPlan* out) {
  for (uint64_t i = 0; i < it.ninst; ++i) {
    const dq_inst& in = it.prog[i];
    if (in.cond_count || in.kind == DQ_MEASURE || in.kind == DQ_RESET || in.kind == DQ_G_UNSUPPORTED)
      return false;
  }
  for (uint32_t l = 0; l < 64; ++l) out->perm[l] = l;
  uint32_t rb = 0;
  if (fused_plan(it.n, it.prog, it.ninst, DQ_SEM_SHOTS, kHbmTB, (int)kHbmM, 0, &out->blob, &out->offs,
                 out->perm, &out->synth, &rb) != DQ_OK ||
      (!out->offs.empty() && rb != kHbmM - kHbmTB)) {
    clear_error();
    return false;
  }
  return true;
}

// Adds a planned HBM item whose state lives at `hbm` (device, 2^n amplitudes)
// and whose sweep programs sit at byte `base` of the set's program blob.
void add_hbm_program(LaunchSet& ls, const HbmPlan& pl, uint64_t base, uint32_t n,
                     uint64_t cbits_off, uint32_t ncbits, double2* hbm) {
  TProg pg{};
  pg.n = n;
  pg.lb = 13;  // reported local bits; the HBM branch sizes its shared memory by hbm_smem
  pg.ncbits = ncbits;
  pg.cbits_off = cbits_off;
  pg.hbm = hbm;
  pg.sweep_first = (uint32_t)ls.sweeps.size();
  pg.nsweeps = (uint32_t)pl.offs.size();
  pg.synth = (long long)pl.synth;
  for (uint64_t off : pl.offs) {
    const uint32_t pb = sweep_prog_bytes(pl.blob.data() + off);
    ls.sweeps.push_back(TSweep{base + off, 1u << (n - kHbmM), sweep_run_bits(pl.blob.data() + off),
                               pb, 0});
    ls.hbm_smem = std::max<size_t>(ls.hbm_smem, sizeof(double2) * (2 * (1u << kHbmM) + kMaxSlots) + pb);
  }
  ls.progs.push_back(pg);
  ls.max_lb = std::max(ls.max_lb, pg.lb);
  ls.max_ncbits = std::max(ls.max_ncbits, ncbits);
}

// Op types whose `mat` indexes the matrix pool (push_mat in encode_gateop).
bool op_uses_pool(uint8_t type) {
  return type == T_ONEQ || type == T_PHASE || type == T_DIAG || type == T_DENSE;
}

// One program's ops and matrices, encoded on its own (matrix offsets into
// its own pool, condition offsets from 0) so that programs can be encoded
// on several host threads and appended to a launch set afterwards.
struct ProgCode {
  std::vector<TOp> ops;
  std::vector<double2> pool;
  int rc = DQ_OK;
  std::string err;
};

void encode_prog_code(const dq_inst* prog, uint64_t ninst, uint32_t n, uint32_t lb, ProgCode& out) {
  Encoded e;
  out.rc = encode_program(prog, ninst, n, 0, e);
  if (out.rc != DQ_OK) {
    out.err = dq_last_error();
    return;
  }
  mark_remote(e.ops.data(), e.ops.size(), lb);
  out.ops = group_phases(e.ops, lb);
  out.pool = std::move(e.pool);
}

// Appends a program encoded by encode_prog_code: the same records add_program
// would write (matrix and condition offsets moved to the set's pools).
int add_prog_code(LaunchSet& ls, const ProgCode& pc, const dq_cond* conds, uint64_t nconds,
                  uint32_t n, uint32_t lb, uint64_t base_seed, uint64_t cbits_off, uint32_t ncbits,
                  double2* state_out) {
  if (pc.rc != DQ_OK) return fail(pc.rc, pc.err);
  TProg pg{};
  pg.ops_off = (uint32_t)ls.enc.ops.size();
  const uint32_t pool_base = (uint32_t)ls.enc.pool.size();
  const uint32_t cond_base = (uint32_t)ls.conds.size();
  for (uint64_t c = 0; c < nconds; ++c) ls.conds.push_back(conds[c]);
  ls.enc.pool.insert(ls.enc.pool.end(), pc.pool.begin(), pc.pool.end());
  for (TOp t : pc.ops) {
    if (op_uses_pool(t.type)) t.mat += pool_base;
    if (t.cond_count) t.cond_first += cond_base;
    ls.enc.ops.push_back(t);
  }
  pg.nops = (uint32_t)pc.ops.size();
  pg.n = n;
  pg.lb = lb;
  pg.ncbits = ncbits;
  pg.base_seed = base_seed;
  pg.cbits_off = cbits_off;
  pg.state_out = state_out;
  ls.progs.push_back(pg);
  ls.max_lb = std::max(ls.max_lb, lb);
  ls.max_ncbits = std::max(ls.max_ncbits, ncbits);
  return DQ_OK;
}

int add_program(LaunchSet& ls, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
                uint64_t nconds, uint32_t n, uint32_t lb, uint64_t base_seed, uint64_t cbits_off,
                uint32_t ncbits, double2* state_out) {
  TProg pg{};
  pg.ops_off = (uint32_t)ls.enc.ops.size();
  const uint32_t cond_base = (uint32_t)ls.conds.size();
  for (uint64_t c = 0; c < nconds; ++c) ls.conds.push_back(conds[c]);
  DQ_TRY(encode_program(prog, ninst, n, cond_base, ls.enc));
  pg.nops = (uint32_t)(ls.enc.ops.size() - pg.ops_off);
  mark_remote(ls.enc.ops.data() + pg.ops_off, pg.nops, lb);
  {
    const std::vector<TOp> tail(ls.enc.ops.begin() + pg.ops_off, ls.enc.ops.end());
    const std::vector<TOp> grouped = group_phases(tail, lb);
    ls.enc.ops.resize(pg.ops_off);
    ls.enc.ops.insert(ls.enc.ops.end(), grouped.begin(), grouped.end());
    pg.nops = (uint32_t)grouped.size();
  }
  pg.n = n;
  pg.lb = lb;
  pg.ncbits = ncbits;
  pg.base_seed = base_seed;
  pg.cbits_off = cbits_off;
  pg.state_out = state_out;
  ls.progs.push_back(pg);
  ls.max_lb = std::max(ls.max_lb, lb);
  ls.max_ncbits = std::max(ls.max_ncbits, ncbits);
  return DQ_OK;
}

// Launch geometry of k_traj: opt-in shared memory, cluster dimension and as
// many clusters as can be resident at once (capped by the item count).
struct TrajLaunch {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  int threads = 256;
  uint32_t clusters = 0;
};

template <int THREADS>
int config_traj_t(uint32_t C, size_t smem, uint64_t nitems, TrajLaunch* L) {
  DQ_CUDA_TRY(cudaFuncSetAttribute(k_traj<THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  L->attr[0].id = cudaLaunchAttributeClusterDimension;
  L->attr[0].val.clusterDim.x = C;
  L->attr[0].val.clusterDim.y = 1;
  L->attr[0].val.clusterDim.z = 1;
  L->cfg.blockDim = dim3(THREADS, 1, 1);
  L->cfg.dynamicSmemBytes = smem;
  L->cfg.attrs = L->attr;
  L->cfg.numAttrs = 1;
  L->cfg.gridDim = dim3(C, 1, 1);
  int max_clusters = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&max_clusters, (void*)k_traj<THREADS>, &L->cfg);
  if (e != cudaSuccess || max_clusters < 1) {
    cudaGetLastError();
    return fail(DQ_ERR_UNSUPPORTED, std::string("trajectory kernel does not fit: cluster of ") +
                                        std::to_string(C) + " CTAs x " + std::to_string(smem) +
                                        " B shared memory");
  }
  uint64_t ncl = std::min<uint64_t>((uint64_t)max_clusters, nitems);
  if (ncl < 1) ncl = 1;
  L->cfg.gridDim = dim3((unsigned)(ncl * C), 1, 1);
  L->threads = THREADS;
  L->clusters = (uint32_t)ncl;
  return DQ_OK;
}

int config_traj(int threads, uint32_t C, size_t smem, uint64_t nitems, TrajLaunch* L) {
  if (threads == 128) return config_traj_t<128>(C, smem, nitems, L);
  if (threads == 256) return config_traj_t<256>(C, smem, nitems, L);
  return config_traj_t<512>(C, smem, nitems, L);
}

int launch_traj(TrajLaunch& L, const TrajParams& P, cudaStream_t st) {
  L.cfg.stream = st;
  L.cfg.attrs = L.attr;
  if (L.threads == 128) DQ_CUDA_TRY(cudaLaunchKernelEx(&L.cfg, k_traj<128>, P));
  else if (L.threads == 256) DQ_CUDA_TRY(cudaLaunchKernelEx(&L.cfg, k_traj<256>, P));
  else DQ_CUDA_TRY(cudaLaunchKernelEx(&L.cfg, k_traj<512>, P));
  return DQ_OK;
}

size_t traj_smem(const LaunchSet& ls) {
  return std::max<size_t>(ls.hbm_smem, sizeof(double2) * (1u << ls.max_lb) + sizeof(double) * 48 +
                                           sizeof(int32_t) * std::max<uint32_t>(ls.max_ncbits, 1));
}

// Device buffers of one launch, freed on scope exit.
struct LaunchBuffers {
  TOp* ops = nullptr;
  double2* pool = nullptr;
  dq_cond* conds = nullptr;
  TProg* progs = nullptr;
  TItem* items = nullptr;
  uint8_t* blob = nullptr;
  TSweep* sweeps = nullptr;
  unsigned long long* ctr = nullptr;  // [0] queue, [1] boundary, [2] failed
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t st = nullptr;
  bool own_st = false;  // destroy st with the buffers
  ~LaunchBuffers() {
    if (st) cudaStreamSynchronize(st);
    if (ops) cudaFree(ops);
    if (pool) cudaFree(pool);
    if (conds) cudaFree(conds);
    if (progs) cudaFree(progs);
    if (items) cudaFree(items);
    if (blob) cudaFree(blob);
    if (sweeps) cudaFree(sweeps);
    if (ctr) cudaFree(ctr);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (own_st && st) cudaStreamDestroy(st);
  }
};

template <class T>
int upload(T** dst, const std::vector<T>& v, cudaStream_t st) {
  const size_t bytes = sizeof(T) * std::max<size_t>(v.size(), 1);
  DQ_CUDA_TRY(cudaMalloc((void**)dst, bytes));
  if (!v.empty())
    DQ_CUDA_TRY(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
  return DQ_OK;
}

// Runs every item of ls in one persistent launch; cbits land in d_cbits.
int run_launch(LaunchSet& ls, int threads, int device, cudaStream_t st, int32_t* d_cbits,
               dq_traj_stats* acc) {
  if (ls.items.empty()) return DQ_OK;
  if (ls.enc.pool.empty()) ls.enc.pool.push_back(make_double2(0, 0));
  LaunchBuffers b;
  b.st = st;
  DQ_TRY(upload(&b.ops, ls.enc.ops, st));
  DQ_TRY(upload(&b.pool, ls.enc.pool, st));
  DQ_TRY(upload(&b.conds, ls.conds, st));
  DQ_TRY(upload(&b.progs, ls.progs, st));
  DQ_TRY(upload(&b.items, ls.items, st));
  if (ls.blob_host) {
    DQ_CUDA_TRY(cudaMalloc((void**)&b.blob, std::max<size_t>(ls.blob_host_bytes, 16)));
    DQ_CUDA_TRY(cudaMemcpyAsync(b.blob, ls.blob_host, ls.blob_host_bytes, cudaMemcpyHostToDevice, st));
  } else {
    DQ_TRY(upload(&b.blob, ls.blob, st));
  }
  DQ_TRY(upload(&b.sweeps, ls.sweeps, st));
  DQ_CUDA_TRY(cudaMalloc((void**)&b.ctr, 3 * sizeof(unsigned long long)));
  const unsigned long long init[3] = {0ULL, 0ULL, 0x7fffffffffffffffULL};
  DQ_CUDA_TRY(cudaMemcpyAsync(b.ctr, init, sizeof(init), cudaMemcpyHostToDevice, st));
  DQ_CUDA_TRY(cudaEventCreate(&b.e0));
  DQ_CUDA_TRY(cudaEventCreate(&b.e1));
  TrajParams P{};
  P.ops = b.ops;
  P.pool = b.pool;
  P.conds = b.conds;
  P.progs = b.progs;
  P.items = b.items;
  P.cbits_out = d_cbits;
  P.queue = b.ctr;
  P.boundary = b.ctr + 1;
  P.failed = reinterpret_cast<long long*>(b.ctr + 2);
  P.nitems = ls.items.size();
  P.sweep_blob = b.blob;
  P.sweeps = b.sweeps;
  (void)device;
  TrajLaunch L;
  DQ_TRY(config_traj(threads, ls.C, traj_smem(ls), P.nitems, &L));
  const uint32_t clusters = L.clusters;
  DQ_CUDA_TRY(cudaEventRecord(b.e0, st));
  DQ_TRY(launch_traj(L, P, st));
  DQ_CUDA_TRY(cudaEventRecord(b.e1, st));
  unsigned long long ctr[3];
  DQ_CUDA_TRY(cudaMemcpyAsync(ctr, b.ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
  DQ_CUDA_TRY(cudaStreamSynchronize(st));
  float ms = 0.f;
  DQ_CUDA_TRY(cudaEventElapsedTime(&ms, b.e0, b.e1));
  acc->boundary_draws += ctr[1];
  const long long f = (long long)ctr[2];
  if (f != 0x7fffffffffffffffLL && (acc->failed_inst < 0 || f < acc->failed_inst))
    acc->failed_inst = f;
  acc->kernel_ms += ms;
  acc->cluster_span = std::max(acc->cluster_span, ls.C);
  acc->clusters = clusters;
  acc->threads = (uint32_t)threads;
  acc->local_bits = std::max(acc->local_bits, ls.max_lb);
  acc->launches += 1;
  return DQ_OK;
}

int check_opts(const dq_traj_opts* opts, int* threads, uint32_t* max_span, uint32_t* force_lb) {
  dq_traj_opts o{};
  if (opts) o = *opts;
  *threads = o.threads ? o.threads : 256;
  if (*threads != 128 && *threads != 256 && *threads != 512)
    return fail(DQ_ERR_INVALID_ARG, "threads must be 128, 256 or 512");
  *max_span = o.max_cluster ? (uint32_t)o.max_cluster : 8u;
  if (*max_span != 1 && *max_span != 2 && *max_span != 4 && *max_span != 8)
    return fail(DQ_ERR_INVALID_ARG, "max_cluster must be 1, 2, 4 or 8");
  *force_lb = 0;
  if (o.local_bits) {
    if (o.local_bits < 1 || (uint32_t)o.local_bits > kLocalBitsMax)
      return fail(DQ_ERR_INVALID_ARG, "local_bits must be in 1..13");
    *force_lb = (uint32_t)o.local_bits;
  }
  return DQ_OK;
}

// Amplitudes per CTA (2^lb) and cluster span for an n-qubit trajectory.
int geometry(uint32_t n, uint32_t max_span, uint32_t force_lb, uint32_t* lb, uint32_t* C) {
  *lb = std::min(n, force_lb ? force_lb : kLocalBitsMax);
  // a smaller max_span needs more amplitudes per CTA than 2^13: not possible
  *C = 1u << (n - *lb);
  if (*C > max_span)
    return fail(DQ_ERR_INVALID_ARG, "a " + std::to_string(n) + "-qubit trajectory needs " +
                                        std::to_string(*C) + " CTAs per cluster, more than max_cluster");
  return DQ_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void init_stats(dq_traj_stats* s) {
  memset(s, 0, sizeof(*s));
  s->failed_inst = -1;
}

}  // namespace
}  // namespace dq

// A trajectory batch captured once as a CUDA graph (seed upload, counter
// reset, the persistent launch, result copies) and replayed per call.
struct dq_traj_plan_s {
  int device = 0;
  uint64_t shots = 0, ncbits = 0;
  dq::LaunchBuffers buf;
  int32_t* d_cbits = nullptr;
  int32_t* h_cbits = nullptr;            // pinned
  uint64_t* h_seed = nullptr;            // pinned: base seed of the next replay
  unsigned long long* h_ctr = nullptr;   // pinned: [0..3) initial, [3..6) results
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  dq::TrajLaunch L;
  dq::TrajParams P{};
  dq_traj_stats geom{};
  ~dq_traj_plan_s() {
    if (buf.st) cudaStreamSynchronize(buf.st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (d_cbits) cudaFree(d_cbits);
    if (h_cbits) cudaFreeHost(h_cbits);
    if (h_seed) cudaFreeHost(h_seed);
    if (h_ctr) cudaFreeHost(h_ctr);
  }
};

using namespace dq;

extern "C" {

int dq_run_trajectories(int device, uint32_t n, const dq_inst* prog, uint64_t ninst,
                        const dq_cond* conds, uint64_t nconds, uint64_t base_seed, uint64_t shot0,
                        uint64_t shots, int32_t* cbits_out, uint64_t ncbits,
                        const dq_traj_opts* opts, dq_traj_stats* stats) {
  dq_traj_stats acc;
  init_stats(&acc);
  if (stats) *stats = acc;
  if (n < 1 || n > kTrajMaxQubits)
    return fail(DQ_ERR_INVALID_ARG, "dq_run_trajectories: n must be in 1..16");
  if (ninst && !prog) return fail(DQ_ERR_INVALID_ARG, "null program");
  if (shots && ncbits && !cbits_out) return fail(DQ_ERR_INVALID_ARG, "null cbits output");
  if (ncbits > kTrajMaxCbits) return fail(DQ_ERR_INVALID_ARG, "at most 1024 classical bits");
  if (shots > (1ULL << 40)) return fail(DQ_ERR_INVALID_ARG, "too many shots");
  for (uint64_t i = 0; i < ninst; ++i) DQ_TRY(validate_inst(prog[i], n, nconds, ncbits, conds, i));
  int threads;
  uint32_t max_span, force_lb, lb, C;
  DQ_TRY(check_opts(opts, &threads, &max_span, &force_lb));
  DQ_TRY(geometry(n, max_span, force_lb, &lb, &C));
  const auto t0 = std::chrono::steady_clock::now();
  LaunchSet ls;
  ls.C = C;
  DQ_TRY(add_program(ls, prog, ninst, conds, nconds, n, lb, base_seed + shot0, 0,
                     (uint32_t)ncbits, nullptr));
  ls.items.resize(shots);
  for (uint64_t s = 0; s < shots; ++s) ls.items[s] = TItem{0, 0, s};
  acc.prepare_ms = ms_since(t0);

  DeviceGuard g(device);
  cudaStream_t st = nullptr;
  DQ_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int32_t* d_out = nullptr;
  const size_t out_bytes = sizeof(int32_t) * (size_t)shots * ncbits;
  int rc = DQ_OK;
  cudaError_t e = cudaMalloc((void**)&d_out, std::max<size_t>(out_bytes, 4));
  if (e != cudaSuccess) rc = fail(DQ_ERR_OOM, std::string("cudaMalloc(cbits): ") + cudaGetErrorString(e));
  if (rc == DQ_OK) rc = run_launch(ls, threads, device, st, d_out, &acc);
  if (rc == DQ_OK && out_bytes) {
    e = cudaMemcpyAsync(cbits_out, d_out, out_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, std::string("copy cbits: ") + cudaGetErrorString(e));
  }
  cudaStreamSynchronize(st);
  if (d_out) cudaFree(d_out);
  cudaStreamDestroy(st);
  if (acc.failed_inst >= 0) acc.failed_inst &= (1LL << 40) - 1;
  if (stats) *stats = acc;
  DQ_TRY(rc);
  if (acc.failed_inst >= 0)
    return fail(DQ_ERR_UNSUPPORTED, "instruction " + std::to_string(acc.failed_inst) +
                                        ": unsupported generic gate reached in a trajectory");
  return DQ_OK;
}

int dq_run_batch(int device, const dq_batch_item* items, uint64_t nitems,
                 const dq_traj_opts* opts, dq_traj_stats* stats) {
  dq_traj_stats acc;
  init_stats(&acc);
  if (stats) *stats = acc;
  if (nitems && !items) return fail(DQ_ERR_INVALID_ARG, "null items");
  int threads;
  uint32_t max_span, force_lb;
  DQ_TRY(check_opts(opts, &threads, &max_span, &force_lb));
  for (uint64_t k = 0; k < nitems; ++k) {
    const dq_batch_item& it = items[k];
    const std::string pre = "item " + std::to_string(k) + ": ";
    if (it.n < 1 || it.n > kMaxQubits) return fail(DQ_ERR_INVALID_ARG, pre + "n must be in 1..34");
    if (it.ninst && !it.prog) return fail(DQ_ERR_INVALID_ARG, pre + "null program");
    if (it.ncbits && !it.cbits_out) return fail(DQ_ERR_INVALID_ARG, pre + "null cbits output");
    if (it.ncbits > kTrajMaxCbits) return fail(DQ_ERR_INVALID_ARG, pre + "at most 1024 classical bits");
    for (uint64_t i = 0; i < it.ninst; ++i) {
      const int rc = validate_inst(it.prog[i], it.n, it.nconds, it.ncbits, it.conds, i);
      if (rc != DQ_OK) return fail(rc, pre + dq_last_error());
    }
  }
  DeviceGuard g(device);
  const auto t0 = std::chrono::steady_clock::now();
  // DQSIM_BATCH_TIMING=1: host phase times on stderr
  static const bool timing = [] {
    const char* e = getenv("DQSIM_BATCH_TIMING");
    return e && atoi(e) != 0;
  }();
  auto tlast = t0;
  auto mark = [&](const char* what) {
    if (!timing) return;
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[dq_run_batch] %-14s %8.3f ms\n", what,
            std::chrono::duration<double, std::milli>(now - tlast).count());
    tlast = now;
  };
  // One persistent launch takes every item it can: states of up to 16 qubits
  // live in a cluster's shared memory; unitary items of 17..30 qubits keep
  // their state in HBM and run as fused tile sweeps by one cluster each.
  // Everything shares one cluster span (the widest any item needs).  Left
  // for separate launches: items whose slice at that span would hold fewer
  // than 16 amplitudes, and every resident item when local_bits is forced
  // (grouped by span); left for the engine (one dq_run each): large items
  // with measurements, resets or conditions.
  std::vector<uint64_t> resident, hbm_items, engine_items, large;
  std::vector<HbmPlan> plans;
  for (uint64_t k = 0; k < nitems; ++k) {
    if (items[k].n <= kTrajMaxQubits) resident.push_back(k);
    else large.push_back(k);
  }
  {
    // plan the large items on host threads
    std::vector<HbmPlan> lp(large.size());
    std::vector<char> ok(large.size(), 0);
    const bool hbm_ok = threads == 256 && !force_lb;
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::max<size_t>(1, std::min<size_t>(hw, large.size()));
    auto work = [&](unsigned t) {
      for (size_t i = t; i < large.size(); i += nt) {
        const dq_batch_item& it = items[large[i]];
        ok[i] = hbm_ok && it.n <= kHbmItemMaxQubits && plan_hbm_item(it, &lp[i]);
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    for (size_t i = 0; i < large.size(); ++i) {
      if (ok[i]) {
        hbm_items.push_back(large[i]);
        plans.push_back(std::move(lp[i]));
      } else {
        engine_items.push_back(large[i]);
      }
    }
  }
  mark("plan large");
  uint32_t Cmain = hbm_items.empty() ? 1u : std::min<uint32_t>(8u, max_span);
  for (uint64_t k : resident) {
    uint32_t lb, C;
    DQ_TRY(geometry(items[k].n, max_span, force_lb, &lb, &C));
    if (!force_lb) Cmain = std::max(Cmain, C);
  }
  const uint32_t cbits_main = (uint32_t)__builtin_ctz(Cmain);
  // set 0: the main launch (span Cmain); sets 1..4: spans 1, 2, 4, 8 for the rest
  LaunchSet sets[5];
  sets[0].C = Cmain;
  for (int c = 0; c < 4; ++c) sets[1 + c].C = 1u << c;
  std::vector<std::vector<uint64_t>> members(5);
  std::vector<uint32_t> item_lb(nitems, 0);
  for (uint64_t k : resident) {
    const uint32_t n = items[k].n;
    uint32_t lb, C;
    geometry(n, max_span, force_lb, &lb, &C);
    if (!force_lb && n >= cbits_main + 4) {
      item_lb[k] = n - cbits_main;
      members[0].push_back(k);
    } else {
      item_lb[k] = lb;
      members[1 + __builtin_ctz(C)].push_back(k);
    }
  }
  for (uint64_t h = 0; h < hbm_items.size(); ++h) members[0].push_back(hbm_items[h]);
  std::vector<int64_t> plan_of(nitems, -1);
  for (uint64_t h = 0; h < hbm_items.size(); ++h) plan_of[hbm_items[h]] = (int64_t)h;
  // HBM item states: one device allocation
  std::vector<uint64_t> hbm_off(hbm_items.size(), 0);
  uint64_t hbm_amps = 0;
  for (uint64_t h = 0; h < hbm_items.size(); ++h) {
    hbm_off[h] = hbm_amps;
    hbm_amps += 1ULL << items[hbm_items[h]].n;
  }
  // per set: state outputs packed into one device buffer, cbits likewise
  struct Out { uint64_t item, state_off, cbits_off; };
  std::vector<Out> outs[5];
  uint64_t state_amps[5] = {0, 0, 0, 0, 0}, cbit_words[5] = {0, 0, 0, 0, 0};
  for (int c = 0; c < 5; ++c) {
    // costliest first (longest-processing-time order for the work queue)
    std::vector<uint64_t>& m = members[c];
    std::stable_sort(m.begin(), m.end(), [&](uint64_t a, uint64_t b) {
      return (items[a].ninst << items[a].n) > (items[b].ninst << items[b].n);
    });
    for (uint64_t k : m) {
      const bool packed = items[k].state_out && plan_of[k] < 0;
      Out o{k, packed ? state_amps[c] : ~0ULL, cbit_words[c]};
      if (packed) state_amps[c] += 1ULL << items[k].n;
      cbit_words[c] += items[k].ncbits;
      outs[c].push_back(o);
    }
  }
  // encode the resident items on host threads (each into its own ops and
  // matrix pool; appended to the launch sets in queue order below)
  std::vector<ProgCode> codes(nitems);
  {
    std::vector<uint64_t> todo;
    for (int c = 0; c < 5; ++c)
      for (const Out& o : outs[c])
        if (plan_of[o.item] < 0) todo.push_back(o.item);
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::max<size_t>(1, std::min<size_t>(hw, todo.size() / 8 + 1));
    auto work = [&](unsigned t) {
      for (size_t i = t; i < todo.size(); i += nt) {
        const uint64_t k = todo[i];
        encode_prog_code(items[k].prog, items[k].ninst, items[k].n, item_lb[k], codes[k]);
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
  }
  // the HBM items' sweep programs, copied on host threads into one pinned
  // staging buffer (recycled across calls) and uploaded with one copy
  std::vector<uint64_t> hbm_blob_off(plans.size(), 0);
  size_t hbm_blob_bytes = 0;
  for (size_t h = 0; h < plans.size(); ++h) {
    hbm_blob_off[h] = hbm_blob_bytes;
    hbm_blob_bytes += (plans[h].blob.size() + 15) / 16 * 16;
  }
  // returned to the pool on every exit path; each set's copies are complete
  // by then (run_launch synchronizes its stream, on errors too)
  struct PinnedStage {
    size_t bytes = 0;
    void* p = nullptr;
    ~PinnedStage() { pinned_free(bytes, p); }
  } stage;
  void* hbm_blob = nullptr;
  if (hbm_blob_bytes) {
    DQ_TRY(pinned_alloc(hbm_blob_bytes, &hbm_blob));
    stage.bytes = hbm_blob_bytes;
    stage.p = hbm_blob;
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::max<size_t>(1, std::min<size_t>(hw, plans.size() / 8 + 1));
    auto work = [&](unsigned t) {
      for (size_t h = t; h < plans.size(); h += nt)
        memcpy(static_cast<uint8_t*>(hbm_blob) + hbm_blob_off[h], plans[h].blob.data(), plans[h].blob.size());
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    sets[0].blob_host = static_cast<const uint8_t*>(hbm_blob);
    sets[0].blob_host_bytes = hbm_blob_bytes;
  }
  acc.prepare_ms = ms_since(t0);
  mark("group+encode");

  cudaStream_t st = nullptr;
  DQ_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = DQ_OK;
  double2* d_hbm = nullptr;
  if (hbm_amps) {
    // from the engine's size-keyed buffer cache: a repeated batch does not
    // pay cudaMalloc/cudaFree of its HBM states
    void* p = nullptr;
    rc = cache_alloc(device, sizeof(double2) * hbm_amps, &p);
    d_hbm = (double2*)p;
  }
  for (int c = 0; c < 5 && rc == DQ_OK; ++c) {
    if (outs[c].empty()) continue;
    double2* d_states = nullptr;
    int32_t* d_cbits = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_states, sizeof(double2) * std::max<uint64_t>(state_amps[c], 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_cbits, sizeof(int32_t) * std::max<uint64_t>(cbit_words[c], 1));
    if (e != cudaSuccess) rc = fail(DQ_ERR_OOM, std::string("cudaMalloc(batch outputs): ") + cudaGetErrorString(e));
    const auto tp = std::chrono::steady_clock::now();
    LaunchSet& ls = sets[c];
    for (const Out& o : outs[c]) {
      if (rc != DQ_OK) break;
      const dq_batch_item& it = items[o.item];
      const uint32_t pi = (uint32_t)ls.progs.size();
      if (plan_of[o.item] >= 0) {
        const uint64_t h = (uint64_t)plan_of[o.item];
        add_hbm_program(ls, plans[h], hbm_blob_off[h], it.n, o.cbits_off, (uint32_t)it.ncbits,
                        d_hbm + hbm_off[h]);
      } else {
        rc = add_prog_code(ls, codes[o.item], it.conds, it.nconds, it.n, item_lb[o.item], it.seed,
                           o.cbits_off, (uint32_t)it.ncbits,
                           o.state_off == ~0ULL ? nullptr : d_states + o.state_off);
      }
      ls.items.push_back(TItem{pi, 0, 0});
    }
    acc.prepare_ms += ms_since(tp);
    mark("encode set");
    const double k0 = acc.kernel_ms;
    if (rc == DQ_OK) rc = run_launch(ls, threads, device, st, d_cbits, &acc);
    if (timing) fprintf(stderr, "[dq_run_batch] kernel         %8.3f ms\n", acc.kernel_ms - k0);
    mark("launch set");
    for (const Out& o : outs[c]) {
      if (rc != DQ_OK) break;
      const dq_batch_item& it = items[o.item];
      e = cudaSuccess;
      if (plan_of[o.item] >= 0) {
        // HBM item: undo its sweeps' qubit relabeling, then copy the state out
        const uint64_t h = (uint64_t)plan_of[o.item];
        if (it.state_out) {
          uint64_t extra = 0;
          rc = materialize_perm(d_hbm + hbm_off[h], it.n, plans[h].perm, st, &extra);
          acc.launches += (uint32_t)extra;
          if (rc != DQ_OK) break;
          e = cudaMemcpyAsync(it.state_out, d_hbm + hbm_off[h], sizeof(double2) << it.n,
                              cudaMemcpyDeviceToHost, st);
        }
      } else if (it.state_out) {
        e = cudaMemcpyAsync(it.state_out, d_states + o.state_off, sizeof(double2) << it.n,
                            cudaMemcpyDeviceToHost, st);
      }
      if (e == cudaSuccess && it.ncbits)
        e = cudaMemcpyAsync(it.cbits_out, d_cbits + o.cbits_off, sizeof(int32_t) * it.ncbits,
                            cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, std::string("copy batch outputs: ") + cudaGetErrorString(e));
    }
    cudaStreamSynchronize(st);
    if (d_states) cudaFree(d_states);
    if (d_cbits) cudaFree(d_cbits);
    mark("outputs");
    if (rc == DQ_OK && acc.failed_inst >= 0) {
      // map (program << 40 | instruction) back to the caller's item index
      const uint64_t pi = (uint64_t)acc.failed_inst >> 40;
      const uint64_t inst = (uint64_t)acc.failed_inst & ((1ULL << 40) - 1);
      acc.failed_inst = (int64_t)((outs[c][pi].item << 40) | inst);
      rc = fail(DQ_ERR_UNSUPPORTED, "item " + std::to_string(outs[c][pi].item) + ", instruction " +
                                        std::to_string(inst) + ": unsupported generic gate");
    }
  }
  if (d_hbm) cache_free(device, sizeof(double2) * hbm_amps, d_hbm);
  acc.hbm_items = (uint32_t)hbm_items.size();
  // large states: the HBM engine, one state per size reused across items
  dq_state_t h = nullptr;
  for (uint64_t k : engine_items) {
    if (rc != DQ_OK) break;
    const dq_batch_item& it = items[k];
    if (h && h->n != it.n) {
      dq_state_destroy(h);
      h = nullptr;
    }
    if (!h) rc = dq_state_create(it.n, device, &h);
    else rc = dq_state_reset(h);
    if (rc != DQ_OK) break;
    std::vector<int32_t> cb(std::max<uint64_t>(it.ncbits, 1), -1);
    dq_run_opts o{};
    o.semantics = DQ_SEM_SHOTS;
    o.exec = DQ_EXEC_FUSED;
    dq_profile prof{};
    const auto te = std::chrono::steady_clock::now();
    rc = dq_run(h, it.prog, it.ninst, it.conds, it.nconds, it.seed, cb.data(), it.ncbits, &o, &prof);
    acc.engine_ms += ms_since(te);
    acc.boundary_draws += prof.boundary_draws;
    if (rc != DQ_OK) {
      acc.failed_inst = (int64_t)((k << 40) | (uint64_t)std::max<int64_t>(prof.failed_inst, 0));
      break;
    }
    if (it.ncbits) memcpy(it.cbits_out, cb.data(), sizeof(int32_t) * it.ncbits);
    if (it.state_out) rc = dq_state_download(h, it.state_out, 1ULL << it.n);
    acc.engine_items += 1;
  }
  if (h) dq_state_destroy(h);
  cudaStreamDestroy(st);
  mark("engine items");
  if (stats) *stats = acc;
  return rc;
}

int dq_traj_plan_create(int device, uint32_t n, const dq_inst* prog, uint64_t ninst,
                        const dq_cond* conds, uint64_t nconds, uint64_t shots, uint64_t ncbits,
                        const dq_traj_opts* opts, dq_traj_plan_t* out) {
  if (!out) return fail(DQ_ERR_INVALID_ARG, "null output plan");
  *out = nullptr;
  if (n < 1 || n > kTrajMaxQubits) return fail(DQ_ERR_INVALID_ARG, "plan: n must be in 1..16");
  if (ninst && !prog) return fail(DQ_ERR_INVALID_ARG, "null program");
  if (ncbits > kTrajMaxCbits) return fail(DQ_ERR_INVALID_ARG, "at most 1024 classical bits");
  if (shots < 1 || shots > (1ULL << 40)) return fail(DQ_ERR_INVALID_ARG, "shots must be in 1..2^40");
  for (uint64_t i = 0; i < ninst; ++i) DQ_TRY(validate_inst(prog[i], n, nconds, ncbits, conds, i));
  int threads;
  uint32_t max_span, force_lb, lb, C;
  DQ_TRY(check_opts(opts, &threads, &max_span, &force_lb));
  DQ_TRY(geometry(n, max_span, force_lb, &lb, &C));
  LaunchSet ls;
  ls.C = C;
  DQ_TRY(add_program(ls, prog, ninst, conds, nconds, n, lb, 0, 0, (uint32_t)ncbits, nullptr));
  ls.items.resize(shots);
  for (uint64_t s = 0; s < shots; ++s) ls.items[s] = TItem{0, 0, s};
  if (ls.enc.pool.empty()) ls.enc.pool.push_back(make_double2(0, 0));

  DeviceGuard g(device);
  dq_traj_plan_t p = new (std::nothrow) dq_traj_plan_s();
  if (!p) return fail(DQ_ERR_OOM, "host allocation failed");
  p->device = device;
  p->shots = shots;
  p->ncbits = ncbits;
  auto bail = [&](int rc) {
    delete p;
    return rc;
  };
  const size_t out_bytes = sizeof(int32_t) * (size_t)shots * ncbits;
  int rc = DQ_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == DQ_OK) {
      cudaGetLastError();
      rc = fail(e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
    }
  };
  cu(cudaStreamCreateWithFlags(&p->buf.st, cudaStreamNonBlocking), "cudaStreamCreate");
  if (rc != DQ_OK) return bail(rc);
  p->buf.own_st = true;
  cudaStream_t st = p->buf.st;
  if ((rc = upload(&p->buf.ops, ls.enc.ops, st)) != DQ_OK) return bail(rc);
  if ((rc = upload(&p->buf.pool, ls.enc.pool, st)) != DQ_OK) return bail(rc);
  if ((rc = upload(&p->buf.conds, ls.conds, st)) != DQ_OK) return bail(rc);
  if ((rc = upload(&p->buf.progs, ls.progs, st)) != DQ_OK) return bail(rc);
  if ((rc = upload(&p->buf.items, ls.items, st)) != DQ_OK) return bail(rc);
  cu(cudaMalloc((void**)&p->buf.ctr, 3 * sizeof(unsigned long long)), "cudaMalloc(counters)");
  cu(cudaMalloc((void**)&p->d_cbits, std::max<size_t>(out_bytes, 4)), "cudaMalloc(cbits)");
  cu(cudaMallocHost((void**)&p->h_cbits, std::max<size_t>(out_bytes, 4)), "cudaMallocHost(cbits)");
  cu(cudaMallocHost((void**)&p->h_seed, sizeof(uint64_t)), "cudaMallocHost(seed)");
  cu(cudaMallocHost((void**)&p->h_ctr, 6 * sizeof(unsigned long long)), "cudaMallocHost(counters)");
  cu(cudaEventCreate(&p->buf.e0), "cudaEventCreate");
  cu(cudaEventCreate(&p->buf.e1), "cudaEventCreate");
  if (rc != DQ_OK) return bail(rc);
  p->h_ctr[0] = 0;
  p->h_ctr[1] = 0;
  p->h_ctr[2] = 0x7fffffffffffffffULL;
  p->h_seed[0] = 0;
  TrajParams& P = p->P;
  P.ops = p->buf.ops;
  P.pool = p->buf.pool;
  P.conds = p->buf.conds;
  P.progs = p->buf.progs;
  P.items = p->buf.items;
  P.cbits_out = p->d_cbits;
  P.queue = p->buf.ctr;
  P.boundary = p->buf.ctr + 1;
  P.failed = reinterpret_cast<long long*>(p->buf.ctr + 2);
  P.nitems = shots;
  if ((rc = config_traj(threads, C, traj_smem(ls), shots, &p->L)) != DQ_OK) return bail(rc);
  cu(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (rc != DQ_OK) return bail(rc);
  // capture: seed -> program table, counters reset, launch, results back
  cu(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  if (rc != DQ_OK) return bail(rc);
  cu(cudaMemcpyAsync(&p->buf.progs[0].base_seed, p->h_seed, sizeof(uint64_t),
                     cudaMemcpyHostToDevice, st), "capture seed copy");
  cu(cudaMemcpyAsync(p->buf.ctr, p->h_ctr, 3 * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                     st), "capture counter reset");
  if (rc == DQ_OK) rc = launch_traj(p->L, P, st);
  if (out_bytes)
    cu(cudaMemcpyAsync(p->h_cbits, p->d_cbits, out_bytes, cudaMemcpyDeviceToHost, st),
       "capture cbits copy");
  cu(cudaMemcpyAsync(p->h_ctr + 3, p->buf.ctr, 3 * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, st), "capture counter copy");
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(st, &graph);
  p->graph = graph;
  cu(ee, "cudaStreamEndCapture");
  if (rc == DQ_OK) cu(cudaGraphInstantiate(&p->exec, p->graph, 0), "cudaGraphInstantiate");
  if (rc != DQ_OK) return bail(rc);
  p->geom.cluster_span = C;
  p->geom.clusters = p->L.clusters;
  p->geom.threads = (uint32_t)threads;
  p->geom.local_bits = lb;
  p->geom.launches = 1;
  *out = p;
  return DQ_OK;
}

int dq_traj_plan_run(dq_traj_plan_t p, uint64_t base_seed, int32_t* cbits_out,
                     dq_traj_stats* stats) {
  if (!p || !p->exec) return fail(DQ_ERR_INVALID_ARG, "null or destroyed plan");
  const size_t out_bytes = sizeof(int32_t) * (size_t)p->shots * p->ncbits;
  if (out_bytes && !cbits_out) return fail(DQ_ERR_INVALID_ARG, "null cbits output");
  DeviceGuard g(p->device);
  cudaStream_t st = p->buf.st;
  p->h_seed[0] = base_seed;
  DQ_CUDA_TRY(cudaEventRecord(p->buf.e0, st));
  DQ_CUDA_TRY(cudaGraphLaunch(p->exec, st));
  DQ_CUDA_TRY(cudaEventRecord(p->buf.e1, st));
  DQ_CUDA_TRY(cudaStreamSynchronize(st));
  float ms = 0.f;
  DQ_CUDA_TRY(cudaEventElapsedTime(&ms, p->buf.e0, p->buf.e1));
  if (out_bytes) memcpy(cbits_out, p->h_cbits, out_bytes);
  dq_traj_stats s = p->geom;
  s.boundary_draws = p->h_ctr[4];
  const long long f = (long long)p->h_ctr[5];
  s.failed_inst = f == 0x7fffffffffffffffLL ? -1 : (f & ((1LL << 40) - 1));
  s.kernel_ms = ms;
  if (stats) *stats = s;
  if (s.failed_inst >= 0)
    return fail(DQ_ERR_UNSUPPORTED, "instruction " + std::to_string(s.failed_inst) +
                                        ": unsupported generic gate reached in a trajectory");
  return DQ_OK;
}

int dq_traj_plan_destroy(dq_traj_plan_t p) {
  if (!p) return DQ_OK;
  DeviceGuard g(p->device);
  delete p;
  return DQ_OK;
}

}  // extern "C"
