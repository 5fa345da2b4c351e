// dq_adjsweep.cu — the adjoint backward pass as fused tile sweeps.
//
// The per-gate backward (dq_adjoint.cu) streams psi and lambda through HBM
// once per gate (64 B per amplitude per gate).  Here a sweep loads a tile of
// 2^m amplitudes of both vectors into shared memory (the tile spans the m
// "local" qubits: bits 0..2 for coalescing plus up to m - 3 chosen ones),
// applies a run of gates in reverse program order to both, reduces every
// gate's gradient terms, and writes the tile back: 64 B per amplitude per
// sweep instead of per gate.  A gate can join the current sweep when
//   * it is diagonal (any qubits: a non-local bit is constant over a tile), or
//   * its non-diagonal qubits (a one-qubit target, both qubits of a dense
//     two-qubit gate) are local — the planner widens the local set up to m.
// Gates of three or more qubits end the sweep and are undone by the exact
// per-gate kernels on both vectors (they carry no trainable parameter).
//
// Ops (all act on psi and lambda; V = U^dagger, D_j = dU/dtheta_j):
//   A_ONE   2x2 on a local target; optional local control mask; optional
//           non-local selector bit choosing between two matrix variants
//           (controlled gates with a non-local control: variant 0 = I).
//   A_TWO   dense 4x4 on two local qubits (rxx, swap-like, psi+-, phi+).
//   A_DIAG  diagonal on up to two qubits, local or not, applied elementwise.
//   A_DRUN  header of a run of 4..64 A_DIAG ops applied in one pass: their
//           gradients from a Walsh-Hadamard transform of conj(lambda) psi,
//           their phases as one quadratic phase polynomial (op_drun).
//   A_PHASE header of 2..16 uncontrolled one-qubit ops on three local bits,
//           applied to 8 amplitudes held in registers per thread (op_phase).
// Gradient terms: Re sum conj(lambda_k) (D_j psi_{k-1}) with psi_{k-1} = V psi_k,
// summed per thread, reduced per warp into shared slots [slot][warp], per CTA
// in warp order, and over CTAs in CTA order by k_adj_slots: deterministic for
// a fixed grid.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "dq_adjsweep.cuh"
#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_gates.hpp"
#include "dq_handle.cuh"

namespace dq {
namespace {

constexpr int kAThreads = 256;
constexpr int kAWarps = kAThreads / 32;
constexpr uint32_t kAMaxLocal = 11;
constexpr uint32_t kALoMin = 3;  // qubits 0..2 stay local: 128-byte runs per tile load
constexpr uint32_t kAMaxOps = 192;
constexpr uint32_t kAMaxSlots = 192;

enum AType : uint8_t { A_ONE = 1, A_TWO = 2, A_DIAG = 3, A_DRUN = 4, A_PHASE = 5 };
constexpr uint32_t kAPhaseOps = 16;  // ops of one register phase
constexpr uint32_t kAPhaseStage = 32;  // phase ops of a sweep staged once per CTA, at most
constexpr uint32_t kAMaxSweepOps = 2 * kAMaxOps;  // ops of a sweep, run and phase headers included
constexpr uint32_t kADiagRun = 64;  // diagonal ops applied in one elementwise pass
constexpr uint32_t kADiagRunMin = 4;  // shorter runs stay single A_DIAG ops

struct AOp {
  uint8_t type;
  uint8_t np;        // derivative matrices (gradient slots) of the op
  uint8_t lt, lt2;   // A_ONE: local target bit; A_TWO: local bits of the 4x4 MSB / LSB
  int8_t sel;        // A_ONE: non-local selector position (-1: none)
  uint8_t skip0;     // A_ONE with selector: variant 0 is the identity with no derivatives
  uint8_t dq[2];     // A_DIAG: qubit encodings (bit 7: local; low 7 bits: local bit or global position)
  uint8_t ndq;       // A_DIAG: 1 or 2 qubits (dq[0] = MSB of the diagonal index)
  uint8_t cnt;       // A_DRUN / A_PHASE: number of ops that follow it
  uint8_t pad[2];
  uint32_t lctrl;    // A_ONE: local control mask (tile offset bits); A_DIAG: run record (pool offset);
                     // A_DRUN: how many of its ops touch a local qubit (those come first)
  uint32_t slot;     // first sweep-local gradient slot
  uint32_t mat;      // offset of the op's matrices in the pool (double2 units)
};
static_assert(sizeof(AOp) == 24, "AOp layout");

struct ASweepHdr {
  uint32_t n, m, nops, nslots;
  uint64_t ntiles;
  uint32_t lpos[kAMaxLocal];  // local bit positions, ascending
  uint32_t npos_cnt;
  uint32_t npos[64];          // non-local bit positions, ascending
  uint32_t phase_ops;         // > 0: every register phase's op data is staged once per CTA
                              // (phase header lctrl = its first PSub); 0: staged per tile
  uint32_t pad;
};

// One sweep of one (psi, lambda) pair in a multi-job launch.
struct AJob {
  double2* psi;
  double2* lam;
  const ASweepHdr* hdr;
  const AOp* ops;
  const double2* pool;
  double* partial;       // [slot][chunk]
  const uint32_t* map;   // sweep-local slot -> index into out
  double* out;           // the pair's gradient slots
  uint32_t nslots, pad;
};

__device__ __forceinline__ double2 cfma2(double2 a, double2 b, double2 acc) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double redot(double2 l, double2 w, double acc) {
  return fma(l.x, w.x, fma(l.y, w.y, acc));
}
__device__ __forceinline__ uint32_t ins0a(uint32_t k, uint32_t p) {
  return ((k >> p) << (p + 1)) | (k & ((1u << p) - 1u));
}

// Shared-memory layout of a tile: element o lives at swz(o).  The low three
// index bits are XORed with a fold of the higher ones, so eight threads whose
// elements differ only in higher bits (register phases over low qubits,
// strided pairs) hit eight different 128-byte bank rows.  A bijection on
// [0, 2^m) for every m.
__device__ __forceinline__ uint32_t swz(uint32_t o) {
  return o ^ (((o >> 3) ^ (o >> 6) ^ (o >> 9)) & 7u);
}

__device__ __forceinline__ void cp_async16a(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// x[e] for a run-time e in 0..3 without indexing a local array
__device__ __forceinline__ double2 sel4(const double2 (&x)[4], uint32_t e) {
  const double2 lo = (e & 1u) ? x[1] : x[0];
  const double2 hi = (e & 1u) ? x[3] : x[2];
  return (e & 2u) ? hi : lo;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NP>
__device__ __forceinline__ void flush_acc(const double (&acc)[4], double* accw, uint32_t slot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const double v = warp_sum_d(acc[j]);
    if (lane == 0) accw[(slot + j) * kAWarps + w] += v;
  }
}

template <int NP>
__device__ __noinline__ void op_one(double2* sp, double2* sl, const AOp& op, const double2* pool, uint32_t m,
                       uint64_t base, double* accw) {
  int var = 0;
  if (op.sel >= 0) var = (int)((base >> op.sel) & 1ULL);
  if (var == 0 && op.skip0) return;
  const double2* mt = pool + op.mat + (uint32_t)var * (4u + 4u * NP);
  double2 v[4], d[NP > 0 ? NP : 1][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = mt[i];
#pragma unroll
  for (int j = 0; j < NP; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) d[j][i] = mt[4 + 4 * j + i];
  // zero-insertion positions: target and local controls, ascending
  uint32_t pos[12];
  int npos = 0;
  uint32_t mask = op.lctrl | (1u << op.lt);
  while (mask) {
    const uint32_t b = __ffs(mask) - 1;
    pos[npos++] = b;
    mask &= mask - 1;
  }
  const uint32_t count = (1u << m) >> npos;
  const uint32_t tb = 1u << op.lt;
  const bool plain = op.lctrl == 0;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t k = threadIdx.x; k < count; k += kAThreads) {
    uint32_t o;
    if (plain) {
      o = ins0a(k, op.lt);
    } else {
      o = k;
      for (int p = 0; p < npos; ++p) o = ins0a(o, pos[p]);
      o |= op.lctrl;
    }
    const uint32_t o1 = swz(o | tb);
    o = swz(o);
    const double2 a0 = sp[o], a1 = sp[o1], b0 = sl[o], b1 = sl[o1];
    const double2 p0 = cfma2(v[1], a1, cmul2(v[0], a0));
    const double2 p1 = cfma2(v[3], a1, cmul2(v[2], a0));
    sp[o] = p0;
    sp[o1] = p1;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const double2 w0 = cfma2(d[j][1], p1, cmul2(d[j][0], p0));
      const double2 w1 = cfma2(d[j][3], p1, cmul2(d[j][2], p0));
      acc[j] = redot(b0, w0, redot(b1, w1, acc[j]));
    }
    sl[o] = cfma2(v[1], b1, cmul2(v[0], b0));
    sl[o1] = cfma2(v[3], b1, cmul2(v[2], b0));
  }
  flush_acc<NP>(acc, accw, op.slot);
}

template <int NP>
__device__ __noinline__ void op_two(double2* sp, double2* sl, const AOp& op, const double2* pool, uint32_t m,
                       double* accw) {
  const double2* mt = pool + op.mat;
  const uint32_t ba = 1u << op.lt, bb = 1u << op.lt2;
  const uint32_t p0 = min((uint32_t)op.lt, (uint32_t)op.lt2), p1 = max((uint32_t)op.lt, (uint32_t)op.lt2);
  const uint32_t count = (1u << m) >> 2;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t k = threadIdx.x; k < count; k += kAThreads) {
    const uint32_t b = ins0a(ins0a(k, p0), p1);
    const uint32_t idx[4] = {swz(b), swz(b | bb), swz(b | ba), swz(b | ba | bb)};
    double2 x[4], y[4], p[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      x[r] = sp[idx[r]];
      y[r] = sl[idx[r]];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 4; ++c) s = cfma2(mt[r * 4 + c], x[c], s);
      p[r] = s;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      sp[idx[r]] = p[r];
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 4; ++c) s = cfma2(mt[r * 4 + c], y[c], s);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double2 w = make_double2(0.0, 0.0);
#pragma unroll
        for (int c = 0; c < 4; ++c) w = cfma2(mt[16 * (j + 1) + r * 4 + c], p[c], w);
        acc[j] = redot(y[r], w, acc[j]);
      }
      sl[idx[r]] = s;
    }
  }
  flush_acc<NP>(acc, accw, op.slot);
}

template <int NP>
__device__ __noinline__ void op_diag(double2* sp, double2* sl, const AOp& op, const double2* pool, uint32_t m,
                        uint64_t base, double* accw) {
  // entry index bits: for each diag qubit, its bit from the tile offset (local)
  // or from the tile base (non-local)
  const double2* mt = pool + op.mat;  // [4 entries: v], then [NP][4]: d
  uint32_t lmask[2] = {0, 0}, fixed = 0;
  for (uint32_t a = 0; a < op.ndq; ++a) {
    const uint32_t e = op.dq[a];
    const uint32_t shift = op.ndq - 1 - a;  // dq[0] is the MSB
    if (e & 0x80u) lmask[a] = 1u << (e & 0x7fu);
    else fixed |= (uint32_t)((base >> (e & 0x7fu)) & 1ULL) << shift;
  }
  double2 v[4], d[NP > 0 ? NP : 1][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = mt[i];
#pragma unroll
  for (int j = 0; j < NP; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) d[j][i] = mt[4 + 4 * j + i];
  const uint32_t L = 1u << m;
  const uint32_t sh0 = op.ndq == 2 ? 1u : 0u;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t o = threadIdx.x; o < L; o += kAThreads) {
    uint32_t e = fixed;
    if (lmask[0] && (o & lmask[0])) e |= 1u << sh0;
    if (lmask[1] && (o & lmask[1])) e |= 1u;
    const uint32_t so = swz(o);
    const double2 a = sp[so], b = sl[so];
    const double2 ve = sel4(v, e);
    const double2 p = cmul2(ve, a);
    sp[so] = p;
#pragma unroll
    for (int j = 0; j < NP; ++j) acc[j] = redot(b, cmul2(sel4(d[j], e), p), acc[j]);
    sl[so] = cmul2(ve, b);
  }
  flush_acc<NP>(acc, accw, op.slot);
}

// One diagonal op of a run, staged in shared memory for the current tile.
// The op's diagonal V over its entry index e = 2 b0 + b1 (b0: the MSB qubit;
// a one-qubit op has b1 = 0) has modulus one, so it is exp(i theta(b0, b1))
// with theta = al + be b0 + ga b1 + de b0 b1.  For this tile each qubit bit
// is a constant (non-local qubit, or absent), a bit of threadIdx.x, or one
// of the three register bits of the run's element layout (o = tid + 256 i).
struct DRec {
  double al, be, ga, de;
  uint32_t k0, k1;  // 0: constant, 1: thread bit, 2: register bit
  uint32_t p0, p1;  // constant value / bit of threadIdx.x / register bit
};

__device__ __forceinline__ void drec_stage(DRec& D, const AOp& op, const double2* pool, uint64_t base) {
  const double2* rec = pool + op.lctrl;
  D.al = rec[0].x;
  D.be = rec[0].y;
  D.ga = rec[1].x;
  D.de = rec[1].y;
  uint32_t k[2] = {0, 0}, p[2] = {0, 0};
  for (uint32_t a = 0; a < op.ndq; ++a) {
    const uint32_t e = op.dq[a];
    if (e & 0x80u) {
      const uint32_t bp = e & 0x7fu;
      k[a] = bp >= 8 ? 2u : 1u;
      p[a] = bp >= 8 ? bp - 8 : bp;
    } else {
      p[a] = (uint32_t)((base >> (e & 0x7fu)) & 1ULL);
    }
  }
  D.k0 = k[0]; D.k1 = k[1];
  D.p0 = p[0]; D.p1 = p[1];
}

__device__ __forceinline__ void gadd(double& g0, double& g1, double& g2, uint32_t r, double v) {
  if (r == 0) g0 += v;
  else if (r == 1) g1 += v;
  else g2 += v;
}

// A run of diagonal ops in one elementwise pass.  Every diagonal entry has
// modulus one, so z = conj(lambda) psi is the same before every op of the
// run and op k's gradient term is
//   Re sum_x z_x w_k[e_k(x)],   w_k = V_k dU_k  (entrywise).
// Expanding w_k in the Walsh basis of its two index bits,
//   w_k[2 b0 + b1] = sum_S what_k[S] (-1)^(b0 S0 + b1 S1),
// turns the sum into four Walsh-Hadamard coefficients of z: a warp takes the
// transform of its own 256 elements over the 8 bits that vary inside it
// (3 register bits, 5 lane bits; the 3 warp bits and non-local bits are
// constants that give a sign), after which each lane serves one op.  The run's
// total phase is exp(i theta(x)) with theta a quadratic polynomial in the
// index bits: each thread folds the ops into its constant, the linear terms of
// its three register bits and their pairwise products, and one sincos per
// element applies it to psi and lambda.  The host writes per op
// rec[0] = (al, be), rec[1] = (ga, de), rec[2 + S] = what[S] at pool + lctrl.
__device__ __noinline__ void op_drun(double2* sp, double2* sl, const AOp& hdr, const AOp* sub,
                                     const double2* pool, uint32_t m, uint64_t base, double* accw,
                                     DRec* ds) {
  const uint32_t cnt = hdr.cnt, nloc = hdr.lctrl;  // ops [nloc, cnt) touch non-local qubits only
  __shared__ double s_tconst;
  for (uint32_t j = threadIdx.x; j < cnt; j += kAThreads) drec_stage(ds[j], sub[j], pool, base);
  __syncthreads();
  const uint32_t L = 1u << m;
  const uint32_t tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  // the tile-constant phase of the ops on non-local qubits: one warp, lanes
  // over the ops, a fixed-order butterfly (read after the barrier below)
  if (w == 0) {
    double t = 0.0;
    for (uint32_t u = nloc + (uint32_t)lane; u < cnt; u += 32) {
      const DRec& D = ds[u];
      t += D.al + (D.p0 ? D.be : 0.0) + (D.p1 ? D.ga : 0.0) + ((D.p0 && D.p1) ? D.de : 0.0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) s_tconst = t;
  }
  if (hdr.np) {
    double2 z[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t o = tid + (uint32_t)i * kAThreads;
      double2 zz = make_double2(0.0, 0.0);
      if (o < L) {
        const uint32_t so = swz(o);
        const double2 a = sp[so], b = sl[so];
        zz = make_double2(fma(b.x, a.x, b.y * a.y), fma(b.x, a.y, -b.y * a.x));
      }
      z[i] = zz;
    }
    // Walsh-Hadamard transform over the register bits, then the lane bits:
    // afterwards lane l, register r holds sum_x z_x (-1)^popc(x & M) over the
    // warp's elements, M = l | r << 8
#pragma unroll
    for (int s = 1; s < 8; s <<= 1)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (!(i & s)) {
          const double2 u = z[i], v = z[i | s];
          z[i] = make_double2(u.x + v.x, u.y + v.y);
          z[i | s] = make_double2(u.x - v.x, u.y - v.y);
        }
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const bool up = (lane & s) != 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const double px = __shfl_xor_sync(0xffffffffu, z[i].x, s);
        const double py = __shfl_xor_sync(0xffffffffu, z[i].y, s);
        z[i] = up ? make_double2(px - z[i].x, py - z[i].y) : make_double2(z[i].x + px, z[i].y + py);
      }
    }
    for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
      const uint32_t j = c0 + (uint32_t)lane;
      double contrib = 0.0;
      uint32_t slot = 0xffffffffu;
      uint32_t src[4] = {0, 0, 0, 0}, reg[4] = {0, 0, 0, 0};
      double2 wh[4];
      if (j < cnt && sub[j].np) {
        const AOp op = sub[j];
        const DRec& D = ds[j];
        slot = op.slot;
        const double2* rec = pool + op.lctrl;
        uint32_t lm[2], rm[2], cv[2];
        const uint32_t kk[2] = {D.k0, D.k1}, pp[2] = {D.p0, D.p1};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          lm[a] = (kk[a] == 1 && pp[a] < 5) ? 1u << pp[a] : 0u;
          rm[a] = kk[a] == 2 ? 1u << pp[a] : 0u;
          cv[a] = kk[a] == 0 ? pp[a] : ((kk[a] == 1 && pp[a] >= 5) ? (tid >> pp[a]) & 1u : 0u);
        }
#pragma unroll
        for (int S = 0; S < 4; ++S) {
          const uint32_t s0 = (uint32_t)S >> 1, s1 = (uint32_t)S & 1u;
          double2 v = rec[2 + S];
          if ((s0 & cv[0]) ^ (s1 & cv[1])) v = make_double2(-v.x, -v.y);
          wh[S] = v;
          src[S] = (s0 ? lm[0] : 0u) | (s1 ? lm[1] : 0u);
          reg[S] = (s0 ? rm[0] : 0u) | (s1 ? rm[1] : 0u);
        }
      } else {
#pragma unroll
        for (int S = 0; S < 4; ++S) wh[S] = make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int S = 0; S < 4; ++S) {
        double2 pz = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const double px = __shfl_sync(0xffffffffu, z[r].x, (int)src[S]);
          const double py = __shfl_sync(0xffffffffu, z[r].y, (int)src[S]);
          if (reg[S] == (uint32_t)r) pz = make_double2(px, py);
        }
        contrib = fma(wh[S].x, pz.x, fma(-wh[S].y, pz.y, contrib));
      }
      // every gate of a sweep has slots of its own, so each lane adds its
      // op's term to the warp's slot directly (one writer per slot and warp)
      if (slot != 0xffffffffu) accw[slot * kAWarps + w] += contrib;
    }
  }
  // the run's phase polynomial for this thread's eight elements (the ops on a
  // local qubit; the others' constant comes from warp 0)
  double T = 0.0, G0 = 0.0, G1 = 0.0, G2 = 0.0, H01 = 0.0, H02 = 0.0, H12 = 0.0;
#pragma unroll 2
  for (uint32_t u = 0; u < nloc; ++u) {
    const DRec& D = ds[u];
    const bool r0 = D.k0 == 2, r1 = D.k1 == 2;
    const bool c0 = D.k0 == 1 ? ((tid >> D.p0) & 1u) != 0 : D.p0 != 0;
    const bool c1 = D.k1 == 1 ? ((tid >> D.p1) & 1u) != 0 : D.p1 != 0;
    if (!r0 && !r1) {
      T += D.al + (c0 ? D.be : 0.0) + (c1 ? D.ga : 0.0) + ((c0 && c1) ? D.de : 0.0);
    } else if (r0 && !r1) {
      T += D.al + (c1 ? D.ga : 0.0);
      gadd(G0, G1, G2, D.p0, D.be + (c1 ? D.de : 0.0));
    } else if (!r0 && r1) {
      T += D.al + (c0 ? D.be : 0.0);
      gadd(G0, G1, G2, D.p1, D.ga + (c0 ? D.de : 0.0));
    } else {
      T += D.al;
      gadd(G0, G1, G2, D.p0, D.be);
      gadd(G0, G1, G2, D.p1, D.ga);
      gadd(H01, H02, H12, D.p0 + D.p1 - 1u, D.de);
    }
  }
  __syncthreads();
  T += s_tconst;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint32_t o = tid + (uint32_t)i * kAThreads;
    if (o < L) {
      double ang = T;
      if (i & 1) ang += G0;
      if (i & 2) ang += G1;
      if (i & 4) ang += G2;
      if ((i & 3) == 3) ang += H01;
      if ((i & 5) == 5) ang += H02;
      if ((i & 6) == 6) ang += H12;
      double sn, cs;
      sincos(ang, &sn, &cs);
      const double2 ph = make_double2(cs, sn);
      const uint32_t so = swz(o);
      sp[so] = cmul2(ph, sp[so]);
      sl[so] = cmul2(ph, sl[so]);
    }
  }
}

// One op of a register phase staged in shared memory.
struct PSub {
  double2 v[4];      // U^dagger
  double2 d[4][4];   // np derivatives in the form D' = dU U^dagger (applied to psi before V)
  uint32_t pb;       // index of the target among the phase bits
  uint32_t vk;       // 0: general V; 1: real V; 2: real diagonal, imaginary off-diagonal
  uint32_t np, slot;
  uint32_t tm[4];    // per derivative: bit 2e / 2e + 1 set if Re / Im of D'[e] is non-zero
};

template <int PB>
__device__ __forceinline__ int pair_lo(int k) {  // k-th index with bit PB clear
  return PB == 0 ? 2 * k : (PB == 1 ? (k & 1) | ((k & 2) << 1) : k);
}

// Re sum over the thread's pairs of conj(lambda) D' psi, term by term of D':
// Re(D'[r][c] conj(l_r) p_c) = Re D' Re(conj(l_r) p_c) - Im D' Im(conj(l_r) p_c),
// skipping the parts of D' that are zero (ry: two real entries, rx: two
// imaginary ones).
template <int PB>
__device__ __forceinline__ double grad_terms(const double2 (&a)[8], const double2 (&b)[8], const double2* dp,
                                             uint32_t tm) {
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int r = e >> 1, c = e & 1;
    if (tm & (1u << (2 * e))) {
      double t[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = pair_lo<PB>(k), j = i | (1 << PB);
        const double2 l = b[r ? j : i], p = a[c ? j : i];
        t[k] = fma(l.x, p.x, l.y * p.y);
      }
      s = fma(dp[e].x, (t[0] + t[1]) + (t[2] + t[3]), s);
    }
    if (tm & (2u << (2 * e))) {
      double t[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = pair_lo<PB>(k), j = i | (1 << PB);
        const double2 l = b[r ? j : i], p = a[c ? j : i];
        t[k] = fma(l.x, p.y, -l.y * p.x);
      }
      s = fma(-dp[e].y, (t[0] + t[1]) + (t[2] + t[3]), s);
    }
  }
  return s;
}

// y = V x on one pair for the three shapes of V
template <int VK>
__device__ __forceinline__ void apply2(const double2* v, double2& x0, double2& x1) {
  const double2 a0 = x0, a1 = x1;
  if (VK == 1) {
    x0 = make_double2(fma(v[1].x, a1.x, v[0].x * a0.x), fma(v[1].x, a1.y, v[0].x * a0.y));
    x1 = make_double2(fma(v[3].x, a1.x, v[2].x * a0.x), fma(v[3].x, a1.y, v[2].x * a0.y));
  } else if (VK == 2) {
    x0 = make_double2(fma(-v[1].y, a1.y, v[0].x * a0.x), fma(v[1].y, a1.x, v[0].x * a0.y));
    x1 = make_double2(fma(v[3].x, a1.x, -v[2].y * a0.y), fma(v[3].x, a1.y, v[2].y * a0.x));
  } else {
    x0 = cfma2(v[1], a1, cmul2(v[0], a0));
    x1 = cfma2(v[3], a1, cmul2(v[2], a0));
  }
}

template <int PB, int VK>
__device__ __forceinline__ void phase_one(double2 (&a)[8], double2 (&b)[8], const PSub& P,
                                          double (&acc)[4]) {
  // gradient terms Re <lambda_k| dU U^dagger |psi_k> from the amplitudes
  // before the op, then psi and lambda both take V = U^dagger
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (q < (int)P.np) acc[q] = grad_terms<PB>(a, b, P.d[q], P.tm[q]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = pair_lo<PB>(k), j = i | (1 << PB);
    apply2<VK>(P.v, a[i], a[j]);
    apply2<VK>(P.v, b[i], b[j]);
  }
}

// One op of a straight-line phase on register bit PB: its gradient term from
// the amplitudes before it, then V on psi and lambda.
template <int VK, int PB>
__device__ __forceinline__ double fast_op(double2 (&a)[8], double2 (&b)[8], const PSub& P) {
  const double acc = grad_terms<PB>(a, b, P.d[0], P.tm[0]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = pair_lo<PB>(k), j = i | (1 << PB);
    apply2<VK>(P.v, a[i], a[j]);
    apply2<VK>(P.v, b[i], b[j]);
  }
  return acc;
}

// A register phase of two or three ops on distinct phase bits PB0 < PB1 (<
// PB2), each with one derivative and the same V shape VK (the encoder sorts
// such ops by target: ops on distinct qubits commute), as straight-line code;
// the ops' warp reductions run after all of them, side by side.
template <int VK, int PB0, int PB1, int PB2>
__device__ __forceinline__ void phase_fast(double2 (&a)[8], double2 (&b)[8], const PSub* ps,
                                           double* accw, int lane, int w) {
  double g0 = fast_op<VK, PB0>(a, b, ps[0]);
  double g1 = fast_op<VK, PB1>(a, b, ps[1]);
  double g2 = 0.0;
  if constexpr (PB2 >= 0) g2 = fast_op<VK, PB2>(a, b, ps[2]);
  g0 = warp_sum_d(g0);
  g1 = warp_sum_d(g1);
  if constexpr (PB2 >= 0) g2 = warp_sum_d(g2);
  if (lane == 0) {
    accw[ps[0].slot * kAWarps + w] += g0;
    accw[ps[1].slot * kAWarps + w] += g1;
    if constexpr (PB2 >= 0) accw[ps[2].slot * kAWarps + w] += g2;
  }
}

template <int VK>
__device__ __forceinline__ void phase_fast_bits(uint32_t form, double2 (&a)[8], double2 (&b)[8],
                                                const PSub* ps, double* accw, int lane, int w) {
  switch (form) {
    case 0: phase_fast<VK, 0, 1, 2>(a, b, ps, accw, lane, w); break;
    case 1: phase_fast<VK, 0, 1, -1>(a, b, ps, accw, lane, w); break;
    case 2: phase_fast<VK, 0, 2, -1>(a, b, ps, accw, lane, w); break;
    default: phase_fast<VK, 1, 2, -1>(a, b, ps, accw, lane, w); break;
  }
}

// The op data of one register phase: threads < cnt fill ps[0 .. cnt).
__device__ __forceinline__ void stage_phase(const AOp& hdr, const AOp* sub, const double2* pool,
                                            PSub* ps) {
  const uint32_t cnt = hdr.cnt;
  const uint32_t pbits[3] = {hdr.lt, hdr.lt2, (uint32_t)hdr.dq[0]};
  if (threadIdx.x < cnt) {
    const AOp op = sub[threadIdx.x];
    PSub& P = ps[threadIdx.x];
    const double2* mt = pool + op.mat;
    P.np = op.np;
    P.slot = op.slot;
    P.pb = op.lt == pbits[0] ? 0u : (op.lt == pbits[1] ? 1u : 2u);
    for (int i = 0; i < 4; ++i) P.v[i] = mt[i];
    const bool real = mt[0].y == 0.0 && mt[1].y == 0.0 && mt[2].y == 0.0 && mt[3].y == 0.0;
    const bool rxl = mt[0].y == 0.0 && mt[3].y == 0.0 && mt[1].x == 0.0 && mt[2].x == 0.0;
    P.vk = real ? 1u : (rxl ? 2u : 0u);
    // D' blocks follow the dU blocks (uncontrolled one-qubit ops only)
    for (uint32_t q = 0; q < op.np; ++q) {
      uint32_t tm = 0;
      for (int i = 0; i < 4; ++i) {
        const double2 dv = mt[4 + 4 * op.np + 4 * q + i];
        P.d[q][i] = dv;
        tm |= (dv.x != 0.0 ? 1u : 0u) << (2 * i);
        tm |= (dv.y != 0.0 ? 2u : 0u) << (2 * i);
      }
      P.tm[q] = tm;
    }
  }
}

// A register phase: every thread holds the 8 amplitudes of psi and lambda
// that differ in the phase's three local bits and applies the phase's
// uncontrolled one-qubit ops (on those bits) in order.  Each op's gradient
// terms are reduced per warp right after the op (all lanes take part: the
// group loop runs the same trip count on every thread).  staged: ps already
// holds the phase's op data (staged once per CTA).
__device__ __noinline__ void op_phase(double2* sp, double2* sl, const AOp& hdr, const AOp* sub,
                                      const double2* pool, uint32_t m, double* accw, PSub* ps,
                                      bool staged) {
  const uint32_t cnt = hdr.cnt;
  const uint32_t pbits[3] = {hdr.lt, hdr.lt2, (uint32_t)hdr.dq[0]};
  if (!staged) {
    stage_phase(hdr, sub, pool, ps);
    __syncthreads();
  }
  const uint32_t groups = (1u << m) >> 3;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t g0 = 0; g0 < groups; g0 += kAThreads) {
    const uint32_t g = g0 + threadIdx.x;
    const bool valid = g < groups;
    const uint32_t ob = ins0a(ins0a(ins0a(valid ? g : 0u, pbits[0]), pbits[1]), pbits[2]);
    // swz is linear over XOR and ob has the phase bits clear, so
    // swz(ob | bits) = swz(ob) ^ swz(bits)
    const uint32_t sb = swz(ob);
    const uint32_t s0 = swz(1u << pbits[0]), s1 = swz(1u << pbits[1]), s2 = swz(1u << pbits[2]);
    auto off = [&](int i) {
      return sb ^ ((i & 1) ? s0 : 0u) ^ ((i & 2) ? s1 : 0u) ^ ((i & 4) ? s2 : 0u);
    };
    double2 a[8], b[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      a[i] = valid ? sp[off(i)] : make_double2(0.0, 0.0);
      b[i] = valid ? sl[off(i)] : make_double2(0.0, 0.0);
    }
    // straight-line form (header pad[0] = 1 + VK * 4 + bit form)
    const uint32_t fast = hdr.pad[0];
    if (fast) {
      const uint32_t vk = (fast - 1u) >> 2, form = (fast - 1u) & 3u;
      if (vk == 1) phase_fast_bits<1>(form, a, b, ps, accw, lane, w);
      else if (vk == 2) phase_fast_bits<2>(form, a, b, ps, accw, lane, w);
      else phase_fast_bits<0>(form, a, b, ps, accw, lane, w);
    }
#pragma unroll 1
    for (uint32_t u = 0; u < (fast ? 0u : cnt); ++u) {
      const PSub& P = ps[u];
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      switch (P.pb * 3 + P.vk) {
        case 0: phase_one<0, 0>(a, b, P, acc); break;
        case 1: phase_one<0, 1>(a, b, P, acc); break;
        case 2: phase_one<0, 2>(a, b, P, acc); break;
        case 3: phase_one<1, 0>(a, b, P, acc); break;
        case 4: phase_one<1, 1>(a, b, P, acc); break;
        case 5: phase_one<1, 2>(a, b, P, acc); break;
        case 6: phase_one<2, 0>(a, b, P, acc); break;
        case 7: phase_one<2, 1>(a, b, P, acc); break;
        default: phase_one<2, 2>(a, b, P, acc); break;
      }
      for (uint32_t q = 0; q < P.np; ++q) {
        const double v = warp_sum_d(acc[q]);
        if (lane == 0) accw[(P.slot + q) * kAWarps + w] += v;
      }
    }
    if (valid) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        sp[off(i)] = a[i];
        sl[off(i)] = b[i];
      }
    }
  }
}

// One backward sweep over tiles t0, t0 + step, ... (< t1) of psi and lambda;
// the CTA's gradient sums go to partial[slot * nparts + part].  Every thread
// of the CTA calls it; the caller separates consecutive calls by a barrier.
__device__ __forceinline__ void adj_sweep_body(double2* __restrict__ psi, double2* __restrict__ lam,
                                               const ASweepHdr* __restrict__ hp,
                                               const AOp* __restrict__ ops,
                                               const double2* __restrict__ pool, double* partial,
                                               uint32_t part, uint32_t nparts, uint64_t t0,
                                               uint64_t t1, uint64_t step) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ ASweepHdr H;
  __shared__ uint64_t hi_tab[1u << (kAMaxLocal - kALoMin)];
  __shared__ DRec drec[kADiagRun];
  __shared__ PSub psub[kAPhaseOps];
  if (threadIdx.x == 0) H = *hp;
  __syncthreads();
  const uint32_t m = H.m, L = 1u << m;
  double2* sp = reinterpret_cast<double2*>(smraw);
  double2* sl = sp + L;
  double* accw = reinterpret_cast<double*>(sl + L);
  // the sweep's ops, and (phase_ops > 0) every register phase's op data, in
  // shared memory for the whole launch
  AOp* sops = reinterpret_cast<AOp*>(accw + ((H.nslots ? H.nslots : 1u) * kAWarps + 1u) / 2u * 2u);
  PSub* psall = reinterpret_cast<PSub*>(sops + (H.nops + 1u) / 2u * 2u);
  for (uint32_t i = threadIdx.x; i < H.nslots * kAWarps; i += kAThreads) accw[i] = 0.0;
  for (uint32_t i = threadIdx.x; i < H.nops; i += kAThreads) sops[i] = ops[i];
  __syncthreads();
  if (H.phase_ops) {
    for (uint32_t i = 0; i < H.nops; ++i) {
      const AOp op = sops[i];
      if (op.type == A_PHASE) stage_phase(op, sops + i + 1, pool, psall + op.lctrl);
      if (op.type == A_PHASE || op.type == A_DRUN) i += op.cnt;
    }
  }
  // offset bits above the 5 contiguous ones -> global bits
  // local bits 0 .. lo_bits-1 are qubits 0 .. lo_bits-1: runs of 2^lo_bits
  // consecutive amplitudes (at least 128 B)
  uint32_t lo_bits = 0;
  while (lo_bits < m && lo_bits < 5 && H.lpos[lo_bits] == lo_bits) ++lo_bits;
  const uint32_t nhi = m - lo_bits;
  for (uint32_t hv = threadIdx.x; hv < (1u << nhi); hv += kAThreads) {
    uint64_t g = 0;
    for (uint32_t b = 0; b < nhi; ++b)
      if (hv >> b & 1u) g |= 1ULL << H.lpos[lo_bits + b];
    hi_tab[hv] = g;
  }
  __syncthreads();
  const uint32_t lo_mask = (1u << lo_bits) - 1u;

  for (uint64_t t = t0; t < t1 && t < H.ntiles; t += step) {
    uint64_t base = 0;
    for (uint32_t b = 0; b < H.npos_cnt; ++b)
      if (t >> b & 1ULL) base |= 1ULL << H.npos[b];
    // all of the tile's copies in flight at once (cp.async straight into the
    // swizzled layout), then one wait
    for (uint32_t o = threadIdx.x; o < L; o += kAThreads) {
      const uint64_t g = base | (o & lo_mask) | hi_tab[o >> lo_bits];
      cp_async16a(sp + swz(o), psi + g);
      cp_async16a(sl + swz(o), lam + g);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    for (uint32_t i = 0; i < H.nops; ++i) {
      const AOp op = sops[i];
      if (op.type == A_DRUN) {
        op_drun(sp, sl, op, sops + i + 1, pool, m, base, accw, drec);
        i += op.cnt;
        __syncthreads();
        continue;
      }
      if (op.type == A_PHASE) {
        op_phase(sp, sl, op, sops + i + 1, pool, m, accw, H.phase_ops ? psall + op.lctrl : psub,
                 H.phase_ops != 0);
        i += op.cnt;
        __syncthreads();
        continue;
      }
      switch (op.type) {
        case A_ONE:
          switch (op.np) {
            case 0: op_one<0>(sp, sl, op, pool, m, base, accw); break;
            case 1: op_one<1>(sp, sl, op, pool, m, base, accw); break;
            case 2: op_one<2>(sp, sl, op, pool, m, base, accw); break;
            case 3: op_one<3>(sp, sl, op, pool, m, base, accw); break;
            default: op_one<4>(sp, sl, op, pool, m, base, accw); break;
          }
          break;
        case A_TWO:
          if (op.np) op_two<1>(sp, sl, op, pool, m, accw);
          else op_two<0>(sp, sl, op, pool, m, accw);
          break;
        default:
          if (op.np) op_diag<1>(sp, sl, op, pool, m, base, accw);
          else op_diag<0>(sp, sl, op, pool, m, base, accw);
          break;
      }
      __syncthreads();
    }
    for (uint32_t o = threadIdx.x; o < L; o += kAThreads) {
      const uint64_t g = base | (o & lo_mask) | hi_tab[o >> lo_bits];
      psi[g] = sp[swz(o)];
      lam[g] = sl[swz(o)];
    }
    __syncthreads();
  }
  for (uint32_t s = threadIdx.x; s < H.nslots; s += kAThreads) {
    double a = 0.0;
    for (int w = 0; w < kAWarps; ++w) a += accw[s * kAWarps + w];
    partial[(size_t)s * nparts + part] = a;
  }
}

__global__ void __launch_bounds__(kAThreads, 2)
    k_adj_sweep(double2* __restrict__ psi, double2* __restrict__ lam, const ASweepHdr* __restrict__ hp,
                const AOp* __restrict__ ops, const double2* __restrict__ pool, double* partial) {
  adj_sweep_body(psi, lam, hp, ops, pool, partial, blockIdx.x, gridDim.x, blockIdx.x, ~0ULL,
                 gridDim.x);
}

// Sweep k of many independent (psi, lambda) pairs in one launch: job j is
// one parameter set's sweep, split into chunks of chunk_tiles consecutive
// tiles; the CTAs take (job, chunk) work items in order.  Chunk c of job j
// writes its sums to jobs[j].partial[slot * nchunks + c].
__global__ void __launch_bounds__(kAThreads, 2)
    k_adj_sweep_multi(const AJob* __restrict__ jobs, uint32_t njobs, uint32_t nchunks,
                      uint64_t chunk_tiles) {
  const uint64_t work = (uint64_t)njobs * nchunks;
  for (uint64_t w = blockIdx.x; w < work; w += gridDim.x) {
    const AJob J = jobs[w / nchunks];
    const uint32_t c = (uint32_t)(w % nchunks);
    adj_sweep_body(J.psi, J.lam, J.hdr, J.ops, J.pool, J.partial, c, nchunks, c * chunk_tiles,
                   (c + 1) * chunk_tiles, 1);
    __syncthreads();
  }
}

// jobs[j].out[map[s]] = sum over chunks (in order) of jobs[j].partial[s][chunk]
__global__ void k_adj_slots_multi(const AJob* __restrict__ jobs, uint32_t nchunks) {
  const AJob J = jobs[blockIdx.y];
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= J.nslots) return;
  double a = 0.0;
  for (uint32_t c = 0; c < nchunks; ++c) a += J.partial[(size_t)s * nchunks + c];
  J.out[J.map[s]] = a;
}

// out[map[s]] = sum over CTAs (in order) of partial[s][cta]
__global__ void k_adj_slots(const double* partial, uint32_t nslots, uint32_t ctas,
                            const uint32_t* map, double* out) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  double a = 0.0;
  for (uint32_t c = 0; c < ctas; ++c) a += partial[(size_t)s * ctas + c];
  out[map[s]] = a;
}

// ---- host planner ----------------------------------------------------------------------------

inline hc cjh(hc z) { return hc{z.re, -z.im}; }

// One gate of the reversed program, classified for the sweep.
struct AGate {
  int64_t inst;
  int kind;  // 0: one-qubit, 1: controlled one-qubit, 2: diagonal (<= 2 qubits), 3: dense 2q, 4: per-gate
  uint32_t t = 0, c = 0;      // target / control (kind 0, 1)
  uint32_t qa = 0, qb = 0;    // diagonal / dense qubits (qa = MSB)
  uint32_t nq = 0;            // diagonal: 1 or 2
  hc u[4];                    // kind 0/1: 2x2 (block)
  hc du[4][4];                // derivatives of the 2x2 (block)
  hc dg[4], ddg[4][4];        // kind 2: diagonal and its derivatives
  hc m4[16], dm4[16];         // kind 3: 4x4 and its derivative
  int np = 0;                 // active derivatives
  uint32_t slot0 = 0;         // first global slot
};

bool diag2(const hc u[4]) { return is_zero(u[1]) && is_zero(u[2]); }

}  // namespace

// Implemented in dq_adjoint.cu: 2x2 block + derivatives of a (controlled)
// one-qubit parametrised kind; derivatives of rxx / rzz.
bool adjoint_block_derivs(const dq_inst& in, hc u[4], hc d[4][4], int* np);
bool adjoint_rxx_rzz_deriv(const dq_inst& in, hc m[16], hc dm[16]);
bool adjoint_controlled_block(int kind);

namespace {

int classify_gate(const dq_inst& in, const int32_t* pidx, uint64_t r, uint32_t slot0, AGate& g) {
  g.inst = (int64_t)r;
  g.slot0 = slot0;
  int active[4] = {0, 0, 0, 0};
  int nact = 0;
  if (pidx)
    for (int j = 0; j < 4; ++j)
      if (pidx[4 * r + j] >= 0) active[nact++] = j;
  hc u[4], d[4][4];
  int np = 0;
  const bool param_block = adjoint_block_derivs(in, u, d, &np);
  if (param_block || matrix_1q(in.kind, in.p, u)) {
    const bool ctl = param_block ? adjoint_controlled_block(in.kind) : false;
    for (int i = 0; i < 4; ++i) g.u[i] = u[i];
    g.np = nact;
    for (int a = 0; a < nact; ++a)
      for (int i = 0; i < 4; ++i) g.du[a][i] = d[active[a]][i];
    // diagonal only if the matrix and every active derivative are (ry(0) is
    // the identity, its derivative is not diagonal) and at most one
    // parameter is active (u3(0, phi, lambda) with both angles trainable
    // stays a 2x2 op, which carries up to four derivatives)
    bool dg = diag2(u) && nact <= 1;
    for (int a = 0; a < nact; ++a) dg = dg && diag2(g.du[a]);
    if (!ctl) {
      g.t = (uint32_t)in.q[0];
      if (dg) {
        g.kind = 2;
        g.nq = 1;
        g.qa = g.t;
        g.dg[0] = u[0];
        g.dg[1] = u[3];
        for (int a = 0; a < nact; ++a) {
          g.ddg[a][0] = g.du[a][0];
          g.ddg[a][1] = g.du[a][3];
        }
      } else {
        g.kind = 0;
      }
      return DQ_OK;
    }
    g.c = (uint32_t)in.q[0];
    g.t = (uint32_t)in.q[1];
    if (dg) {  // controlled diagonal: a two-qubit diagonal (c = MSB)
      g.kind = 2;
      g.nq = 2;
      g.qa = g.c;
      g.qb = g.t;
      g.dg[0] = R(1); g.dg[1] = R(1); g.dg[2] = u[0]; g.dg[3] = u[3];
      for (int a = 0; a < nact; ++a) {
        g.ddg[a][0] = R(0); g.ddg[a][1] = R(0);
        g.ddg[a][2] = g.du[a][0]; g.ddg[a][3] = g.du[a][3];
      }
    } else {
      g.kind = 1;
    }
    return DQ_OK;
  }
  if (nact > 0 && !(in.kind == DQ_RXX || in.kind == DQ_RZZ))
    return fail(DQ_ERR_INTERNAL, "parameter slot on a kind without a derivative");
  Gate gt;
  if (!matrix_nq(in, gt)) return fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
  if (gt.k > 2) {
    g.kind = 4;
    return DQ_OK;
  }
  hc dm[16];
  for (int i = 0; i < 16; ++i) dm[i] = R(0);
  if (nact) adjoint_rxx_rzz_deriv(in, gt.m, dm);
  g.np = nact;
  GateOp op;
  classify(gt, op);
  g.qa = gt.qubits[0];
  g.qb = gt.qubits[1];
  if (nact == 0 && (op.cls == GC_ONE_Q || op.cls == GC_PHASE || op.cls == GC_XPERM)) {
    // controlled one-qubit without a trainable parameter (rxx / rzz at
    // special angles with an active slot keep their 4x4 and derivative)
    g.c = gt.qubits[0];
    g.t = gt.qubits[1];
    for (int i = 0; i < 4; ++i) g.u[i] = hc{0, 0};
    g.u[0] = gt.m[10]; g.u[1] = gt.m[11]; g.u[2] = gt.m[14]; g.u[3] = gt.m[15];
    if (diag2(g.u)) {
      g.kind = 2;
      g.nq = 2;
      g.qa = g.c;
      g.qb = g.t;
      g.dg[0] = R(1); g.dg[1] = R(1); g.dg[2] = g.u[0]; g.dg[3] = g.u[3];
    } else {
      g.kind = 1;
    }
    return DQ_OK;
  }
  bool dgn = true;
  for (int r2 = 0; r2 < 4; ++r2)
    for (int c2 = 0; c2 < 4; ++c2)
      if (r2 != c2 && (!is_zero(gt.m[r2 * 4 + c2]) || (nact && !is_zero(dm[r2 * 4 + c2]))))
        dgn = false;
  if (dgn) {
    g.kind = 2;
    g.nq = 2;
    for (int i = 0; i < 4; ++i) {
      g.dg[i] = gt.m[i * 5];
      if (nact) g.ddg[0][i] = dm[i * 5];
    }
    return DQ_OK;
  }
  g.kind = 3;
  for (int i = 0; i < 16; ++i) {
    g.m4[i] = gt.m[i];
    g.dm4[i] = dm[i];
  }
  return DQ_OK;
}

struct ASweepPlan {
  uint64_t Lmask = 0;
  std::vector<AGate> gates;  // reverse program order
};

// Qubits a gate needs local.
uint64_t need_local(const AGate& g) {
  switch (g.kind) {
    case 0: case 1: return 1ULL << g.t;
    case 3: return (1ULL << g.qa) | (1ULL << g.qb);
    default: return 0;
  }
}

void push_mats(std::vector<double2>& pool, const hc* m, int count) {
  for (int i = 0; i < count; ++i) pool.push_back(make_double2(m[i].re, m[i].im));
}

// D' = dU V (V = U^dagger, both 2x2 row-major): the derivative in the form
// that acts on the amplitudes before the op.  Parts below 1e-14 of the
// largest are rounding residue of exact zeros (ry: dU V = -i Y / 2) and are
// stored as zeros, which the register phases skip.
void push_dprime(std::vector<double2>& pool, const hc du[4], const hc v[4]) {
  hc d[4];
  double mx = 0.0;
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 2; ++c) {
      const hc x = du[2 * r] * v[c] + du[2 * r + 1] * v[2 + c];
      d[2 * r + c] = x;
      mx = std::max(mx, std::max(std::fabs(x.re), std::fabs(x.im)));
    }
  for (hc& x : d) {
    if (std::fabs(x.re) <= 1e-14 * mx) x.re = 0.0;
    if (std::fabs(x.im) <= 1e-14 * mx) x.im = 0.0;
  }
  push_mats(pool, d, 4);
}

// The record op_drun reads for a diagonal op: the angle polynomial of its
// entries V[2 b0 + b1] = exp(i (al + be b0 + ga b1 + de b0 b1)) and the Walsh
// coefficients what[2 S0 + S1] = 1/4 sum_e V[e] dU[e] (-1)^(b0 S0 + b1 S1).
// A one-qubit diagonal (entry index b0) is the same with b1 = 0: its
// coefficients with S1 = 1 vanish.
void push_drun_record(std::vector<double2>& pool, const hc v[4], const hc dd[4], uint32_t nq) {
  double th[4];
  hc w[4];
  for (int e = 0; e < 4; ++e) {
    const int src = nq == 2 ? e : (e >> 1);
    th[e] = std::atan2(v[src].im, v[src].re);
    w[e] = hc{v[src].re * dd[src].re - v[src].im * dd[src].im, v[src].re * dd[src].im + v[src].im * dd[src].re};
  }
  pool.push_back(make_double2(th[0], th[2] - th[0]));
  pool.push_back(make_double2(th[1] - th[0], th[3] - th[2] - th[1] + th[0]));
  for (int S = 0; S < 4; ++S) {
    double re = 0.0, im = 0.0;
    for (int e = 0; e < 4; ++e) {
      const bool neg = (((e >> 1) & (S >> 1)) ^ (e & S & 1)) != 0;
      re += neg ? -w[e].re : w[e].re;
      im += neg ? -w[e].im : w[e].im;
    }
    pool.push_back(make_double2(0.25 * re, 0.25 * im));
  }
}

// Encodes one sweep's ops given its final local set.
int encode_asweep(const ASweepPlan& sp, uint32_t n, ASweepHdr& hdr, std::vector<AOp>& ops,
                  std::vector<double2>& pool, std::vector<uint32_t>& slot_map) {
  memset(&hdr, 0, sizeof(hdr));
  hdr.n = n;
  uint32_t lidx[64];
  uint32_t m = 0;
  for (uint32_t q = 0; q < n; ++q) {
    if (sp.Lmask >> q & 1ULL) {
      lidx[q] = m;
      hdr.lpos[m++] = q;
    } else {
      hdr.npos[hdr.npos_cnt++] = q;
    }
  }
  hdr.m = m;
  hdr.ntiles = 1ULL << (n - m);
  uint32_t slot = 0;
  for (const AGate& g : sp.gates) {
    AOp op{};
    op.np = (uint8_t)g.np;
    op.slot = slot;
    op.sel = -1;
    op.mat = (uint32_t)pool.size();
    for (int a = 0; a < g.np; ++a) slot_map.push_back(g.slot0 + (uint32_t)a);
    slot += (uint32_t)g.np;
    if (g.kind == 0 || g.kind == 1) {
      op.type = A_ONE;
      op.lt = (uint8_t)lidx[g.t];
      const hc v[4] = {cjh(g.u[0]), cjh(g.u[2]), cjh(g.u[1]), cjh(g.u[3])};
      if (g.kind == 1 && !(sp.Lmask >> g.c & 1ULL)) {
        // non-local control: variant 0 (control 0) is the identity
        op.sel = (int8_t)g.c;
        op.skip0 = 1;
        const hc id[4] = {R(1), R(0), R(0), R(1)};
        push_mats(pool, id, 4);
        for (int a = 0; a < g.np; ++a) {
          const hc z[4] = {R(0), R(0), R(0), R(0)};
          push_mats(pool, z, 4);
        }
      } else if (g.kind == 1) {
        op.lctrl = 1u << lidx[g.c];
      }
      push_mats(pool, v, 4);
      for (int a = 0; a < g.np; ++a) push_mats(pool, g.du[a], 4);
      if (g.kind == 0)
        for (int a = 0; a < g.np; ++a) push_dprime(pool, g.du[a], v);
    } else if (g.kind == 3) {
      op.type = A_TWO;
      op.lt = (uint8_t)lidx[g.qa];
      op.lt2 = (uint8_t)lidx[g.qb];
      hc v[16];
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) v[r * 4 + c] = cjh(g.m4[c * 4 + r]);
      push_mats(pool, v, 16);
      if (g.np) push_mats(pool, g.dm4, 16);
    } else {
      op.type = A_DIAG;
      op.ndq = (uint8_t)g.nq;
      const uint32_t qs[2] = {g.qa, g.qb};
      for (uint32_t a = 0; a < g.nq; ++a)
        op.dq[a] = (sp.Lmask >> qs[a] & 1ULL) ? (uint8_t)(0x80u | lidx[qs[a]]) : (uint8_t)qs[a];
      hc v[4] = {R(1), R(1), R(1), R(1)};
      const uint32_t D = 1u << g.nq;
      for (uint32_t i = 0; i < D; ++i) v[i] = cjh(g.dg[i]);
      push_mats(pool, v, 4);
      hc dd[4] = {R(0), R(0), R(0), R(0)};
      if (g.np > 1) return fail(DQ_ERR_INTERNAL, "diagonal op with more than one derivative");
      if (g.np) {
        for (uint32_t i = 0; i < D; ++i) dd[i] = g.ddg[0][i];
        push_mats(pool, dd, 4);
      }
      op.lctrl = (uint32_t)pool.size();
      push_drun_record(pool, v, dd, g.nq);
    }
    ops.push_back(op);
  }
  // register phases: maximal runs (two or more) of uncontrolled one-qubit ops
  // whose targets fit three local bits; diagonal ops end a phase and go to
  // the diagonal runs, which apply them far more cheaply
  if (m >= 3) {
    std::vector<AOp> phased;
    size_t i = 0;
    while (i < ops.size()) {
      const AOp& o = ops[i];
      const bool one = o.type == A_ONE && o.lctrl == 0 && o.sel < 0;
      if (!one) {
        phased.push_back(ops[i++]);
        continue;
      }
      uint32_t bits[3];
      uint32_t nb = 0;
      size_t j = i;
      uint32_t nones = 0;
      while (j < ops.size() && j - i < kAPhaseOps) {
        const AOp& q = ops[j];
        if (!(q.type == A_ONE && q.lctrl == 0 && q.sel < 0)) break;
        bool have = false;
        for (uint32_t b = 0; b < nb; ++b) have = have || bits[b] == q.lt;
        if (!have) {
          if (nb == 3) break;
          bits[nb++] = q.lt;
        }
        ++nones;
        ++j;
      }
      if (nones < 2) {  // a single op: the plain one-qubit pass
        for (size_t k = i; k < j; ++k) phased.push_back(ops[k]);
        i = j;
        continue;
      }
      // three distinct phase bits: fill with other local bits
      for (uint32_t b = 0; nb < 3 && b < m; ++b) {
        bool have = false;
        for (uint32_t c = 0; c < nb; ++c) have = have || bits[c] == b;
        if (!have) bits[nb++] = b;
      }
      std::sort(bits, bits + 3);
      AOp h{};
      h.type = A_PHASE;
      h.cnt = (uint8_t)(j - i);
      h.lt = (uint8_t)bits[0];
      h.lt2 = (uint8_t)bits[1];
      h.dq[0] = (uint8_t)bits[2];
      std::vector<AOp> run(ops.begin() + (ptrdiff_t)i, ops.begin() + (ptrdiff_t)j);
      // Straight-line form: two or three ops on distinct qubits, one derivative
      // each, one V shape.  Such ops commute, so they are sorted by target bit
      // and the kernel runs them with compile-time register bits.
      {
        auto vk_of = [&](const AOp& q) -> int {
          const double2* mt = pool.data() + q.mat;
          const bool real = mt[0].y == 0.0 && mt[1].y == 0.0 && mt[2].y == 0.0 && mt[3].y == 0.0;
          const bool rxl = mt[0].y == 0.0 && mt[3].y == 0.0 && mt[1].x == 0.0 && mt[2].x == 0.0;
          return real ? 1 : (rxl ? 2 : 0);
        };
        bool fast = (run.size() == 2 || run.size() == 3) && nones == run.size();
        uint32_t distinct = 0;
        for (size_t a = 0; a < run.size(); ++a) {
          bool dup = false;
          for (size_t b2 = 0; b2 < a; ++b2) dup = dup || run[b2].lt == run[a].lt;
          if (!dup) ++distinct;
          fast = fast && run[a].np == 1 && vk_of(run[a]) == vk_of(run[0]);
        }
        fast = fast && distinct == run.size();
        if (fast) {
          std::sort(run.begin(), run.end(), [](const AOp& x, const AOp& y) { return x.lt < y.lt; });
          uint32_t pb[3] = {0, 0, 0};
          for (size_t a = 0; a < run.size(); ++a)
            for (uint32_t b2 = 0; b2 < 3; ++b2)
              if (bits[b2] == run[a].lt) pb[a] = b2;
          int form = -1;
          if (run.size() == 3) form = 0;
          else if (pb[0] == 0 && pb[1] == 1) form = 1;
          else if (pb[0] == 0 && pb[1] == 2) form = 2;
          else if (pb[0] == 1 && pb[1] == 2) form = 3;
          if (form >= 0) h.pad[0] = (uint8_t)(1 + vk_of(run[0]) * 4 + form);
        }
      }
      phased.push_back(h);
      for (const AOp& q : run) phased.push_back(q);
      i = j;
    }
    ops.swap(phased);
  }
  // runs of consecutive diagonal ops become one A_DRUN header + the ops
  std::vector<AOp> grouped;
  for (size_t i = 0; i < ops.size();) {
    if (ops[i].type == A_PHASE) {
      const size_t e = i + 1 + ops[i].cnt;
      for (; i < e; ++i) grouped.push_back(ops[i]);
      continue;
    }
    if (ops[i].type != A_DIAG) {
      grouped.push_back(ops[i++]);
      continue;
    }
    size_t j = i;
    while (j < ops.size() && ops[j].type == A_DIAG && j - i < kADiagRun) ++j;
    if (j - i >= kADiagRunMin) {
      AOp h{};
      h.type = A_DRUN;
      h.cnt = (uint8_t)(j - i);
      for (size_t k = i; k < j; ++k) h.np = (uint8_t)(h.np | (ops[k].np ? 1 : 0));
      // ops on a local qubit first, ops on non-local qubits only (a constant
      // phase over a tile) last; diagonal ops commute.  lctrl = how many
      // touch a local qubit.
      auto local = [](const AOp& o) {
        bool l = false;
        for (uint32_t a = 0; a < o.ndq; ++a) l = l || (o.dq[a] & 0x80u) != 0;
        return l;
      };
      std::stable_partition(ops.begin() + (ptrdiff_t)i, ops.begin() + (ptrdiff_t)j, local);
      uint32_t nloc = 0;
      for (size_t k = i; k < j; ++k) nloc += local(ops[k]) ? 1u : 0u;
      h.lctrl = nloc;
      grouped.push_back(h);
    }
    for (size_t k = i; k < j; ++k) grouped.push_back(ops[k]);
    i = j;
  }
  ops.swap(grouped);
  // register phases' op data staged once per CTA when it fits
  uint32_t pops = 0;
  for (size_t i = 0; i < ops.size(); ++i)
    if (ops[i].type == A_PHASE) pops += ops[i].cnt;
  if (pops <= kAPhaseStage) {
    uint32_t b = 0;
    for (size_t i = 0; i < ops.size(); ++i)
      if (ops[i].type == A_PHASE) {
        ops[i].lctrl = b;
        b += ops[i].cnt;
      }
    hdr.phase_ops = pops;
  }
  hdr.nops = (uint32_t)ops.size();
  hdr.nslots = slot;
  if (hdr.nops > kAMaxSweepOps) return fail(DQ_ERR_INTERNAL, "too many ops in an adjoint sweep");
  return DQ_OK;
}

// Dynamic shared memory of a sweep: psi and lambda tiles, per-warp gradient
// slots, the op list and the staged phase data (layout as in k_adj_sweep).
size_t asweep_smem(uint32_t m, uint32_t nslots, uint32_t nops, uint32_t phase_ops) {
  const size_t slots = ((size_t)(nslots ? nslots : 1) * kAWarps + 1) / 2 * 2;
  const size_t nops2 = ((size_t)nops + 1) / 2 * 2;
  return sizeof(double2) * 2 * (1u << m) + sizeof(double) * slots + sizeof(AOp) * nops2 +
         sizeof(PSub) * phase_ops;
}

int sweep_ctas(int device) {
  static std::mutex mu;
  static int per_sm[64];
  std::lock_guard<std::mutex> lk(mu);
  if (per_sm[device & 63] == 0) {
    const size_t smem_max = asweep_smem(kAMaxLocal, kAMaxSlots, kAMaxSweepOps, kAPhaseStage);
    DQ_CUDA_TRY(cudaFuncSetAttribute(k_adj_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_max));
    int b = 1;
    DQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_adj_sweep, kAThreads, smem_max));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    per_sm[device & 63] = std::max(1, b) * sms;
  }
  return per_sm[device & 63];
}

// Segments of the backward pass in backward order: fused sweeps and the
// instructions undone one at a time (three or more qubits).
struct BackSeg {
  bool sweep;
  ASweepPlan plan;
  int64_t inst;
};

int plan_backward_segments(uint32_t n, const dq_inst* prog, uint64_t ninst, const int32_t* pidx,
                           uint64_t nslots, std::vector<BackSeg>& segs) {
  // global slot numbering: program order, parameter order within a gate
  std::vector<uint32_t> first_slot(ninst + 1, 0);
  for (uint64_t i = 0; i < ninst; ++i) {
    uint32_t c = 0;
    if (pidx)
      for (int j = 0; j < 4; ++j) c += pidx[4 * i + j] >= 0;
    first_slot[i + 1] = first_slot[i] + c;
  }
  if (first_slot[ninst] != nslots) return fail(DQ_ERR_INTERNAL, "slot count mismatch");
  const uint32_t m_max = std::min<uint32_t>(n, kAMaxLocal);
  const uint32_t lo = std::min<uint32_t>(n, kALoMin);
  const uint64_t lo_mask = (1ULL << lo) - 1;
  ASweepPlan cur;
  cur.Lmask = lo_mask;
  uint32_t cur_slots = 0;
  auto close = [&]() {
    if (!cur.gates.empty()) {
      // widen the local set to m_max with the lowest unused qubits (more
      // work per tile, fewer tiles; the set only needs to contain the gates')
      for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(cur.Lmask) < m_max; ++q)
        cur.Lmask |= 1ULL << q;
      segs.push_back(BackSeg{true, cur, -1});
    }
    cur = ASweepPlan();
    cur.Lmask = lo_mask;
    cur_slots = 0;
  };
  for (uint64_t r = ninst; r-- > 0;) {
    const dq_inst& in = prog[r];
    if (in.kind == DQ_ID || in.kind == DQ_U0 || in.kind == DQ_BARRIER || in.kind == DQ_CLASSICAL ||
        in.kind == DQ_G_NOOP)
      continue;
    AGate g;
    DQ_TRY(classify_gate(in, pidx, r, first_slot[r], g));
    if (g.kind == 4) {
      close();
      segs.push_back(BackSeg{false, ASweepPlan(), (int64_t)r});
      continue;
    }
    const uint64_t need = need_local(g);
    const uint64_t widened = cur.Lmask | need;
    if ((uint32_t)__builtin_popcountll(widened) > m_max || cur.gates.size() >= kAMaxOps ||
        cur_slots + (uint32_t)g.np > kAMaxSlots) {
      close();
    }
    cur.Lmask |= need;
    cur.gates.push_back(g);
    cur_slots += (uint32_t)g.np;
  }
  close();
  return DQ_OK;
}

}  // namespace

int adjoint_backward_fused(double2* psi, double2* lam, uint32_t n, const dq_inst* prog,
                           uint64_t ninst, const int32_t* pidx, uint64_t nslots, double* d_slots,
                           cudaStream_t st, int device, AdjSweepStats* stats) {
  using Seg = BackSeg;
  std::vector<Seg> segs;
  DQ_TRY(plan_backward_segments(n, prog, ninst, pidx, nslots, segs));
  const int ctas_max = sweep_ctas(device);
  if (ctas_max <= 0) return DQ_ERR_CUDA;
  // device buffers for all sweeps at once
  std::vector<ASweepHdr> hdrs;
  std::vector<AOp> ops;
  std::vector<double2> pool;
  std::vector<uint32_t> slot_map;
  struct SweepRef {
    size_t hdr, op0, slot0;
    uint32_t nslots;
    unsigned grid;
  };
  std::vector<SweepRef> refs;
  size_t max_partial = 1;
  for (const Seg& s : segs) {
    if (!s.sweep) continue;
    ASweepHdr hdr;
    const size_t op0 = ops.size(), sl0 = slot_map.size();
    std::vector<AOp> o;
    DQ_TRY(encode_asweep(s.plan, n, hdr, o, pool, slot_map));
    for (AOp& a : o) ops.push_back(a);
    const unsigned grid = (unsigned)std::min<uint64_t>(hdr.ntiles, (uint64_t)ctas_max);
    refs.push_back(SweepRef{hdrs.size(), op0, sl0, hdr.nslots, grid});
    max_partial = std::max(max_partial, (size_t)hdr.nslots * grid);
    hdrs.push_back(hdr);
  }
  if (pool.empty()) pool.push_back(make_double2(0, 0));
  if (slot_map.empty()) slot_map.push_back(0);
  if (ops.empty()) ops.push_back(AOp{});
  if (hdrs.empty()) hdrs.push_back(ASweepHdr{});
  ASweepHdr* d_hdr = nullptr;
  AOp* d_ops = nullptr;
  double2* d_pool = nullptr;
  uint32_t* d_map = nullptr;
  double* d_part = nullptr;
  int rc = DQ_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == DQ_OK) {
      cudaGetLastError();
      rc = fail(e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
    }
  };
  cu(pool_malloc_async((void**)&d_hdr, sizeof(ASweepHdr) * hdrs.size(), st), "cudaMallocAsync(hdr)");
  cu(pool_malloc_async((void**)&d_ops, sizeof(AOp) * ops.size(), st), "cudaMallocAsync(ops)");
  cu(pool_malloc_async((void**)&d_pool, sizeof(double2) * pool.size(), st), "cudaMallocAsync(pool)");
  cu(pool_malloc_async((void**)&d_map, sizeof(uint32_t) * slot_map.size(), st), "cudaMallocAsync(map)");
  cu(pool_malloc_async((void**)&d_part, sizeof(double) * max_partial, st), "cudaMallocAsync(partials)");
  if (rc == DQ_OK) {
    cu(cudaMemcpyAsync(d_hdr, hdrs.data(), sizeof(ASweepHdr) * hdrs.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_ops, ops.data(), sizeof(AOp) * ops.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_pool, pool.data(), sizeof(double2) * pool.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_map, slot_map.data(), sizeof(uint32_t) * slot_map.size(), cudaMemcpyHostToDevice, st), "copy");
  }
  size_t si = 0;
  uint64_t sweeps = 0, pergate = 0;
  for (const Seg& s : segs) {
    if (rc != DQ_OK) break;
    if (!s.sweep) {
      GateOp op;
      const dq_inst& in = prog[s.inst];
      hc u4[4];
      (void)u4;
      Gate gt;
      if (!matrix_nq(in, gt)) {
        rc = fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
        break;
      }
      const uint32_t D = 1u << gt.k;
      std::vector<hc> t(gt.m, gt.m + D * D);
      for (uint32_t r = 0; r < D; ++r)
        for (uint32_t c = 0; c < D; ++c) gt.m[r * D + c] = cjh(t[c * D + r]);
      classify(gt, op);
      rc = launch_gate(psi, n, op, st, device, nullptr);
      if (rc == DQ_OK) rc = launch_gate(lam, n, op, st, device, nullptr);
      ++pergate;
      continue;
    }
    const SweepRef& ref = refs[si++];
    const ASweepHdr& hdr = hdrs[ref.hdr];
    const size_t smem = asweep_smem(hdr.m, hdr.nslots, hdr.nops, hdr.phase_ops);
    k_adj_sweep<<<ref.grid, kAThreads, smem, st>>>(psi, lam, d_hdr + ref.hdr, d_ops + ref.op0, d_pool,
                                                    d_part);
    cu(cudaGetLastError(), "k_adj_sweep");
    if (ref.nslots && rc == DQ_OK) {
      k_adj_slots<<<(ref.nslots + 127) / 128, 128, 0, st>>>(d_part, ref.nslots, ref.grid,
                                                            d_map + ref.slot0, d_slots);
      cu(cudaGetLastError(), "k_adj_slots");
    }
    ++sweeps;
  }
  if (d_hdr) cudaFreeAsync(d_hdr, st);
  if (d_ops) cudaFreeAsync(d_ops, st);
  if (d_pool) cudaFreeAsync(d_pool, st);
  if (d_map) cudaFreeAsync(d_map, st);
  if (d_part) cudaFreeAsync(d_part, st);
  if (stats) {
    stats->sweeps = sweeps;
    stats->pergate = pergate;
  }
  return rc;
}

// ---- many parameter sets at once -------------------------------------------------------

int adjoint_backward_plan_set(uint32_t n, const dq_inst* prog, uint64_t ninst, const int32_t* pidx,
                              uint64_t nslots, ABatchSet* out) {
  std::vector<BackSeg> segs;
  DQ_TRY(plan_backward_segments(n, prog, ninst, pidx, nslots, segs));
  ABatchSet s;
  for (const BackSeg& g : segs) {
    if (!g.sweep)
      return fail(DQ_ERR_UNSUPPORTED, "a gate of three or more qubits: no batched backward sweep");
    ASweepHdr hdr;
    std::vector<AOp> o;
    const size_t op0 = s.ops.size() / sizeof(AOp), sl0 = s.map.size();
    DQ_TRY(encode_asweep(g.plan, n, hdr, o, s.pool, s.map));
    s.ops.insert(s.ops.end(), reinterpret_cast<const uint8_t*>(o.data()),
                 reinterpret_cast<const uint8_t*>(o.data() + o.size()));
    s.op0.push_back(op0);
    s.slot0.push_back(sl0);
    s.nslots.push_back(hdr.nslots);
    s.hdrs.insert(s.hdrs.end(), reinterpret_cast<const uint8_t*>(&hdr),
                  reinterpret_cast<const uint8_t*>(&hdr + 1));
  }
  if (s.pool.empty()) s.pool.push_back(make_double2(0, 0));
  *out = std::move(s);
  return DQ_OK;
}

int adjoint_backward_batch(double2* const* psi, double2* const* lam, const std::vector<ABatchSet>& sets,
                           double* const* d_slots, cudaStream_t st, int device, uint64_t* launches) {
  const size_t B = sets.size();
  if (!B) return DQ_OK;
  // every set's headers, ops, pools and slot maps in four device arrays
  std::vector<ASweepHdr> hdrs;
  std::vector<AOp> ops;
  std::vector<double2> pool;
  std::vector<uint32_t> map;
  std::vector<size_t> bh(B), bo(B), bp(B), bm(B);
  size_t kmax = 0;
  for (size_t b = 0; b < B; ++b) {
    const ABatchSet& s = sets[b];
    bh[b] = hdrs.size();
    bo[b] = ops.size();
    bp[b] = pool.size();
    bm[b] = map.size();
    for (size_t k = 0; k < s.sweeps(); ++k) {
      ASweepHdr x;
      memcpy(&x, s.hdrs.data() + k * sizeof(ASweepHdr), sizeof(x));
      hdrs.push_back(x);
    }
    const size_t nops = s.ops.size() / sizeof(AOp);
    ops.resize(bo[b] + nops);
    if (nops) memcpy(ops.data() + bo[b], s.ops.data(), nops * sizeof(AOp));
    pool.insert(pool.end(), s.pool.begin(), s.pool.end());
    map.insert(map.end(), s.map.begin(), s.map.end());
    kmax = std::max(kmax, s.sweeps());
  }
  if (hdrs.empty()) return DQ_OK;
  if (ops.empty()) ops.push_back(AOp{});
  if (map.empty()) map.push_back(0);
  const int ctas = sweep_ctas(device);
  if (ctas <= 0) return DQ_ERR_CUDA;
  const uint64_t ntiles = hdrs[0].ntiles;
  const uint64_t chunk_tiles = std::max<uint64_t>(1, std::min<uint64_t>(64, ntiles));
  const uint32_t nchunks = (uint32_t)((ntiles + chunk_tiles - 1) / chunk_tiles);
  // jobs of every sweep index (device pointers filled in once the arrays exist)
  std::vector<AJob> jobs;
  std::vector<size_t> job_hdr, job_ops, job_pool, job_map;
  std::vector<size_t> job0(kmax + 1, 0);
  std::vector<size_t> smem(kmax, 0);
  std::vector<uint32_t> maxsl(kmax, 0);
  size_t part_per_job = 1;
  for (const ASweepHdr& h : hdrs) part_per_job = std::max<size_t>(part_per_job, (size_t)h.nslots * nchunks);
  for (size_t k = 0; k < kmax; ++k) {
    job0[k] = jobs.size();
    for (size_t b = 0; b < B; ++b) {
      const ABatchSet& s = sets[b];
      if (k >= s.sweeps()) continue;
      const ASweepHdr& h = hdrs[bh[b] + k];
      if (h.ntiles != ntiles) return fail(DQ_ERR_INTERNAL, "batched sweeps of unequal tile counts");
      AJob j{};
      j.psi = psi[b];
      j.lam = lam[b];
      j.out = d_slots[b];
      j.nslots = s.nslots[k];
      jobs.push_back(j);
      job_hdr.push_back(bh[b] + k);
      job_ops.push_back(bo[b] + s.op0[k]);
      job_pool.push_back(bp[b]);
      job_map.push_back(bm[b] + s.slot0[k]);
      smem[k] = std::max(smem[k], asweep_smem(h.m, h.nslots, h.nops, h.phase_ops));
      maxsl[k] = std::max(maxsl[k], h.nslots);
    }
  }
  job0[kmax] = jobs.size();
  size_t max_jobs = 1;
  for (size_t k = 0; k < kmax; ++k) max_jobs = std::max(max_jobs, job0[k + 1] - job0[k]);
  ASweepHdr* d_hdr = nullptr;
  AOp* d_ops = nullptr;
  double2* d_pool = nullptr;
  uint32_t* d_map = nullptr;
  double* d_part = nullptr;
  AJob* d_jobs = nullptr;
  int rc = DQ_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == DQ_OK) {
      cudaGetLastError();
      rc = fail(e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
    }
  };
  // the device arrays come from the engine's size-keyed buffer cache: an
  // optimiser loop repeats their sizes, so its steps pay no cudaMalloc/cudaFree
  std::vector<std::pair<void*, size_t>> owned;
  auto take = [&](void** p, size_t bytes) {
    if (rc != DQ_OK) return;
    bytes = std::max<size_t>(bytes, 16);
    const int r = cache_alloc(device, bytes, p);
    if (r != DQ_OK) {
      rc = r;
      *p = nullptr;
      return;
    }
    owned.push_back({*p, bytes});
  };
  take((void**)&d_hdr, sizeof(ASweepHdr) * hdrs.size());
  take((void**)&d_ops, sizeof(AOp) * ops.size());
  take((void**)&d_pool, sizeof(double2) * pool.size());
  take((void**)&d_map, sizeof(uint32_t) * map.size());
  take((void**)&d_part, sizeof(double) * part_per_job * max_jobs);
  take((void**)&d_jobs, sizeof(AJob) * std::max<size_t>(jobs.size(), 1));
  if (rc == DQ_OK) {
    for (size_t k = 0; k < kmax; ++k)
      for (size_t i = job0[k]; i < job0[k + 1]; ++i) {
        AJob& j = jobs[i];
        j.hdr = d_hdr + job_hdr[i];
        j.ops = d_ops + job_ops[i];
        j.pool = d_pool + job_pool[i];
        j.map = d_map + job_map[i];
        j.partial = d_part + (i - job0[k]) * part_per_job;
      }
    cu(cudaMemcpyAsync(d_hdr, hdrs.data(), sizeof(ASweepHdr) * hdrs.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_ops, ops.data(), sizeof(AOp) * ops.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_pool, pool.data(), sizeof(double2) * pool.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_map, map.data(), sizeof(uint32_t) * map.size(), cudaMemcpyHostToDevice, st), "copy");
    cu(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(AJob) * jobs.size(), cudaMemcpyHostToDevice, st), "copy");
  }
  {
    static std::mutex mu;
    static uint64_t attr_done = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!((attr_done >> (device & 63)) & 1ULL)) {
      const size_t smem_max = asweep_smem(kAMaxLocal, kAMaxSlots, kAMaxSweepOps, kAPhaseStage);
      cu(cudaFuncSetAttribute(k_adj_sweep_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_max), "cudaFuncSetAttribute");
      attr_done |= 1ULL << (device & 63);
    }
  }
  for (size_t k = 0; k < kmax && rc == DQ_OK; ++k) {
    const uint32_t nj = (uint32_t)(job0[k + 1] - job0[k]);
    if (!nj) continue;
    const uint64_t work = (uint64_t)nj * nchunks;
    const unsigned grid = (unsigned)std::min<uint64_t>(work, (uint64_t)ctas);
    k_adj_sweep_multi<<<grid, kAThreads, smem[k], st>>>(d_jobs + job0[k], nj, nchunks, chunk_tiles);
    cu(cudaGetLastError(), "k_adj_sweep_multi");
    if (launches) ++*launches;
    if (maxsl[k] && rc == DQ_OK) {
      k_adj_slots_multi<<<dim3((maxsl[k] + 127) / 128, nj), 128, 0, st>>>(d_jobs + job0[k], nchunks);
      cu(cudaGetLastError(), "k_adj_slots_multi");
      if (launches) ++*launches;
    }
  }
  cudaStreamSynchronize(st);
  for (auto& o : owned) cache_free(device, o.second, o.first);
  return rc;
}

}  // namespace dq
