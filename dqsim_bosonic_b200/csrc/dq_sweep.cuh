// dq_sweep.cuh — device side of the fused tile sweep: the encoded sweep
// program layout, the per-op register arithmetic and the per-CTA tile loop
// (sweep_tiles).  Included by the sweep kernel (dq_fused.cu) and by the
// persistent batch kernel (dq_traj.cu), which runs the sweeps of large batch
// items with the CTAs of one cluster.
//
// Kernel geometry.  A tile holds 2^m amplitudes (m = TB + RB local qubits,
// RB = register bits per thread, m <= 12, 64 KiB of FP64 complex at m = 12).
// Local bit k of a tile is physical qubit local_pos[k] (ascending); the tile
// is made of runs of consecutive amplitudes (see SwHeader::run_bits) that a
// warp moves with coalesced cp.async copies.  In shared memory the element
// index is XOR-swizzled (low 3 bits ^= a linear function of the high bits)
// so that any 7 of the 12 local bits can serve as thread bits without bank
// conflicts.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dq_common.cuh"

namespace dq {
namespace {

// Thread geometry: TB thread bits (5 lane + TB-5 warp bits), 2^TB threads per
// CTA.  TB = 7: 128 threads, two CTAs per SM (their phases overlap); TB = 8:
// 256 threads, one CTA per SM.
constexpr int kMaxTB = 8;
constexpr int kMaxM = 12;
constexpr int kMaxSlots = 128;
// bytes of one sweep program (staged in shared memory next to two tile buffers)
// Largest staged sweep program for a tile of 2^m amplitudes: what is left of
// shared memory next to two tile buffers at the CTAs per SM the geometry runs.
__host__ __device__ constexpr int max_prog(int m) { return m >= 12 ? 64 * 1024 : 40 * 1024; }

enum : uint32_t { OP_U1 = 0, OP_U1R, OP_U1X, OP_U2, OP_FLUSH_R, OP_FLUSH_T, OP_GPHASE, OP_U1H,
                  OP_SCALE, OP_HPHASE };

// swizzle vectors of local bits 3..11 (bits 0..2 map to themselves)
__host__ __device__ constexpr uint32_t swz_g(int k) {
  return k == 3 ? 3u : k == 4 ? 5u : k == 5 ? 6u : k == 6 ? 7u : k == 7 ? 3u : k == 8 ? 5u
       : k == 9 ? 6u : k == 10 ? 7u : k == 11 ? 1u : 0u;
}
__host__ __device__ constexpr uint32_t swz_vec(int k) { return k < 3 ? (1u << k) : swz_g(k); }
__host__ __device__ constexpr uint32_t swz(uint32_t e) {
  uint32_t g = 0;
  for (int k = 3; k < kMaxM; ++k)
    if ((e >> k) & 1u) g ^= swz_g(k);
  return e ^ g;
}

// ---- sweep program layout (copied verbatim into shared memory) ----------------
// A tile is made of runs of 2^run_bits consecutive amplitudes (run_bits = 5:
// local bits 0..4 are qubits 0..4, 512-byte runs; run_bits = 3: only qubits
// 0..2 are pinned, 128-byte runs, two more tile qubits free for the gates).
constexpr int kMinRunBits = 3;
constexpr int kMaxRuns = 1 << (kMaxM - kMinRunBits);

struct SwHeader {
  uint32_t m, rb, nphase, nslots;
  uint32_t local_pos[kMaxM];
  uint32_t off_phase, off_op, off_slot, off_slotent;
  uint32_t off_data, prog_bytes;
  uint32_t tile_xload;         // XORed into every tile-load address: X gates opening the sweep
  uint32_t run_bits;           // 5 or 3
  // 2^(m - run_bits) entries each, stored after the header:
  uint32_t off_runoff;         // u64 physical offset of run r (local bits run_bits..m-1 = r)
  uint32_t off_runswz;         // u32 swizzled shared-memory index of run r's first element
  uint32_t flags;              // SWF_* (host side: kernel choice)
  uint32_t off_gstore;         // SwGStore of the last phase (0: none)
};
// Global offsets for the last phase to write its amplitudes straight to the
// state (present when the phase's lanes 0..2 are local bits 0..2, i.e. each
// 8-lane group writes one 128-byte run): element j of thread (lane, warp) is
// at tile base + glane[lane] + gwarp[warp] + sum of gV[b] over the bits b of j.
struct SwGStore {
  uint64_t glane[32];
  uint64_t gwarp[8];
  uint64_t gV[4];
};
// every phase of the sweep is an H phase (OP_HPHASE): the launch may use the
// kernel built with the H-phase path only
constexpr uint32_t SWF_HONLY = 1u;
// every op of the sweep is a one-qubit op without a flush (OP_U1, OP_U1R,
// OP_U1X; controls allowed): the launch may use the kernel built with that
// part of the interpreter only
constexpr uint32_t SWF_UONLY = 2u;
// every phase of the sweep is a straight-line phase (OP_HPHASE) of real 2x2
// sub-ops only: the launch may use the build with that path only
constexpr uint32_t SWF_RONLY = 4u;
// Builds of the tile loop: the whole op interpreter, Hadamard-pattern
// straight-line phases only, plain one-qubit ops only, real-2x2 straight-line
// phases only.
enum : int { FORM_ALL = 0, FORM_H = 1, FORM_U = 2, FORM_R = 3 };
struct SwPhase {
  uint32_t lanesw[32];         // swizzled local index of the lane bits (thread bits 0..4)
  uint32_t warpsw[8];          // swizzled local index of the warp bits (thread bits 5..7)
  uint32_t V[4];               // swizzled local index of each register bit
  uint32_t op_begin, op_end;
  uint32_t xload;              // XORed into every load address: X gates folded into the load
  uint32_t pad1;
};
// 32 bytes, read as two 128-bit words: w0 = type | b0 << 8 | b1 << 16 | creg << 24,
// w1 = ctl_thr | flags << 8 | slot << 16, data = first DATA entry, cnl = non-local controls
struct SwOp {
  uint32_t w0, w1, data, pad;
  uint64_t cnl, pad2;
};
struct SwSlot {
  uint32_t count, start, pad0, pad1;
  double2 w0;
};
struct SwSlotEnt {
  uint64_t mask, pad;
  double2 w;
};
static_assert(sizeof(SwHeader) % 16 == 0 && sizeof(SwPhase) % 16 == 0 && sizeof(SwGStore) % 16 == 0,
              "layout");
static_assert(sizeof(SwOp) % 16 == 0 && sizeof(SwSlot) % 16 == 0 && sizeof(SwSlotEnt) % 16 == 0,
              "layout");

// FLUSH flags: thread-partner tables present (32 lane + 8 warp factors), then
// a register-partner table (2^(RB-1) entries for a register target, 2^RB for
// a thread target).
constexpr uint32_t FL_THR = 1u;
constexpr uint32_t FL_REG = 2u;
constexpr uint32_t FL_PRE = 4u;   // 1q op: flush its target first (data = 4 matrix entries, then flush tables)
// U1H op inside an H phase: its register-partner table depends only on the
// register bits below its target (entries 0 .. 2^b0 - 1 hold every value)
constexpr uint32_t FL_LOWF = 8u;
// OP_HPHASE marks a phase whose ops are K = b1 uncontrolled Hadamard-pattern
// or real 2x2 ops (OP_U1H, OP_U1R) on register bits 0, 1, ..., K-1 in that
// order, optionally followed by the deferred OP_SCALE when the last op is a
// Hadamard (flags bit 0 set, data = the scale): the kernel runs them as
// straight-line code instead of interpreting them.
constexpr uint32_t HPH_SCALE = 1u;

// ---- device helpers -------------------------------------------------------------------

// Hide a value's provenance from the optimiser so that addresses are
// recomputed instead of being kept live (in registers) across a phase.
__device__ __forceinline__ uint32_t opaque(uint32_t x) {
  asm volatile("" : "+r"(x));
  return x;
}
__device__ __forceinline__ uint64_t opaque64(uint64_t x) {
  asm volatile("" : "+l"(x));
  return x;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One-qubit op on register bit B, optionally preceded by the flush of B
// (amplitudes with bit B set times W * F[compress(j)]).  KIND: 0 general
// 2x2, 1 real 2x2, 2 [[1,1],[1,-1]], 3 X.  Controls only occur without a
// pre-flush (the planner fuses flushes into uncontrolled ops only).
// PRE: 0 no flush; 1 flush by the per-thread factor W; 2 flush by W times the
// register-partner table F (known at compile time, no per-pair select).
template <int RB, int B, int KIND, int PRE>
__device__ __forceinline__ void u1_op(double2 (&a)[1 << RB], const double2* __restrict__ D,
                                      uint32_t creg, double2 W, const double2* __restrict__ F) {
  double2 u00, u01, u10, u11;
  if (KIND <= 1) {
    u00 = D[0]; u01 = D[1]; u10 = D[2]; u11 = D[3];
  }
#pragma unroll
  for (int j = 0; j < (1 << RB); ++j) {
    if (j & (1 << B)) continue;
    if (PRE == 0 && (j & creg) != creg) continue;
    const int k = j | (1 << B);
    const double2 x = a[j];
    double2 y = a[k];
    if (PRE == 2) {
      const int idx = ((k >> (B + 1)) << B) | (k & ((1 << B) - 1));
      y = cmul_f(y, cmul_f(W, F[idx]));
    } else if (PRE == 1) {
      y = cmul_f(y, W);
    }
    if (KIND == 0) {
      a[j] = cmac2_f(u00, x, u01, y);
      a[k] = cmac2_f(u10, x, u11, y);
    } else if (KIND == 1) {
      a[j] = make_double2(fma(u00.x, x.x, u01.x * y.x), fma(u00.x, x.y, u01.x * y.y));
      a[k] = make_double2(fma(u10.x, x.x, u11.x * y.x), fma(u10.x, x.y, u11.x * y.y));
    } else if (KIND == 2) {
      a[j] = make_double2(x.x + y.x, x.y + y.y);
      a[k] = make_double2(x.x - y.x, x.y - y.y);
    } else {
      a[j] = y;
      a[k] = x;
    }
  }
}

// dense 4x4 on register bits B0 (MSB of the gate index) and B1
template <int RB, int B0, int B1>
__device__ __forceinline__ void u2_gen(double2 (&a)[1 << RB], const double2* __restrict__ D,
                                       uint32_t creg) {
#pragma unroll
  for (int j = 0; j < (1 << RB); ++j) {
    if (j & ((1 << B0) | (1 << B1))) continue;
    if ((j & creg) != creg) continue;
    const int i0 = j, i1 = j | (1 << B1), i2 = j | (1 << B0), i3 = j | (1 << B0) | (1 << B1);
    const double2 v0 = a[i0], v1 = a[i1], v2 = a[i2], v3 = a[i3];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double2 s01 = cmac2_f(D[4 * r], v0, D[4 * r + 1], v1);
      const double2 s23 = cmac2_f(D[4 * r + 2], v2, D[4 * r + 3], v3);
      const double2 w = make_double2(s01.x + s23.x, s01.y + s23.y);
      if (r == 0) a[i0] = w;
      else if (r == 1) a[i1] = w;
      else if (r == 2) a[i2] = w;
      else a[i3] = w;
    }
  }
}

// flush on register bit B: a[j] *= W * F[compress(j)] for j with bit B set
template <int RB, int B>
__device__ __forceinline__ void flush_reg(double2 (&a)[1 << RB], double2 W,
                                          const double2* __restrict__ F) {
#pragma unroll
  for (int j = 0; j < (1 << RB); ++j) {
    if (!(j & (1 << B))) continue;
    if (F) {
      const int idx = ((j >> (B + 1)) << B) | (j & ((1 << B) - 1));
      a[j] = cmul_f(a[j], cmul_f(W, F[idx]));
    } else {
      a[j] = cmul_f(a[j], W);
    }
  }
}

#define DQ_SW_CASES1(FN, ...)                                          \
  switch (b0) {                                                        \
    case 0: FN<RB, 0>(__VA_ARGS__); break;                             \
    case 1: if (RB > 1) FN<RB, (RB > 1 ? 1 : 0)>(__VA_ARGS__); break;  \
    case 2: if (RB > 2) FN<RB, (RB > 2 ? 2 : 0)>(__VA_ARGS__); break;  \
    case 3: if (RB > 3) FN<RB, (RB > 3 ? 3 : 0)>(__VA_ARGS__); break;  \
    default: break;                                                    \
  }

#define DQ_SW_U1(KIND, PRE)                                                                  \
  switch (b0) {                                                                              \
    case 0: u1_op<RB, 0, KIND, PRE>(a, D, creg, W, F); break;                                \
    case 1: if (RB > 1) u1_op<RB, (RB > 1 ? 1 : 0), KIND, PRE>(a, D, creg, W, F); break;     \
    case 2: if (RB > 2) u1_op<RB, (RB > 2 ? 2 : 0), KIND, PRE>(a, D, creg, W, F); break;     \
    case 3: if (RB > 3) u1_op<RB, (RB > 3 ? 3 : 0), KIND, PRE>(a, D, creg, W, F); break;     \
    default: break;                                                                          \
  }

template <int RB>
__device__ __forceinline__ void u2_dispatch(double2 (&a)[1 << RB], uint32_t b0, uint32_t b1,
                                            uint32_t creg, const double2* __restrict__ D) {
#define DQ_U2C(X, Y)                                                                      \
  if (b0 == X && b1 == Y) {                                                               \
    if (RB > X && RB > Y) u2_gen<RB, (RB > X ? X : 0), (RB > Y ? Y : 1)>(a, D, creg);     \
    return;                                                                               \
  }
  DQ_U2C(0, 1) DQ_U2C(0, 2) DQ_U2C(0, 3) DQ_U2C(1, 2) DQ_U2C(1, 3) DQ_U2C(2, 3)
#undef DQ_U2C
}

// ---- H phases: straight-line Hadamard-pattern ops ---------------------------------------
// Op on register bit B: the upper amplitude y of each pair is multiplied by
// its flush factor (PRE 1: W; PRE 2: W * F[idx], the W * F products formed
// once per distinct F entry: 2^B of them when LOWF), then the butterfly
// (x + y', x - y').  SC: the phase's deferred scale s folds into this op as
// (s x + y', s x - y') with s already in W (PRE 0: y' = s y).
template <int RB, int B, int PRE, bool LOWF, bool SC, bool REAL = false>
__device__ __forceinline__ void hph_op(double2 (&a)[1 << RB], double2 W, const double2* __restrict__ F,
                                       double s, const double2* __restrict__ U = nullptr) {
  double u00 = 0.0, u01 = 0.0, u10 = 0.0, u11 = 0.0;
  if constexpr (REAL) {
    u00 = U[0].x; u01 = U[1].x; u10 = U[2].x; u11 = U[3].x;
  }
  // real ops form each pair's W * F on the spot (fewer live registers next to
  // their matrix)
  constexpr int NF = (PRE == 2 && !REAL) ? (LOWF ? (1 << B) : (1 << (RB - 1))) : 1;
  double2 WF[NF];
  if (PRE == 2 && !REAL) {
#pragma unroll
    for (int i = 0; i < NF; ++i) WF[i] = cmul_f(W, F[i]);
  }
#pragma unroll
  for (int j = 0; j < (1 << RB); ++j) {
    if (j & (1 << B)) continue;
    const int k = j | (1 << B);
    const double2 x = a[j];
    double2 y = a[k];
    if (PRE == 2) {
      const int idx = LOWF ? (k & ((1 << B) - 1)) : (((k >> (B + 1)) << B) | (k & ((1 << B) - 1)));
      if constexpr (REAL) y = cmul_f(y, cmul_f(W, F[idx]));
      else y = cmul_f(y, WF[idx]);
    } else if (PRE == 1) {
      y = cmul_f(y, W);
    } else if (SC) {
      y = make_double2(y.x * s, y.y * s);
    }
    if constexpr (REAL) {  // real 2x2 (same arithmetic as u1_op's KIND 1)
      a[j] = make_double2(fma(u00, x.x, u01 * y.x), fma(u00, x.y, u01 * y.y));
      a[k] = make_double2(fma(u10, x.x, u11 * y.x), fma(u10, x.y, u11 * y.y));
    } else if (SC) {
      a[j] = make_double2(fma(x.x, s, y.x), fma(x.y, s, y.y));
      a[k] = make_double2(fma(x.x, s, -y.x), fma(x.y, s, -y.y));
    } else {
      a[j] = make_double2(x.x + y.x, x.y + y.y);
      a[k] = make_double2(x.x - y.x, x.y - y.y);
    }
  }
}

template <int RB, int B, bool SC, bool REAL = false>
__device__ __forceinline__ void hph_flags(double2 (&a)[1 << RB], uint32_t fl, double2 W,
                                          const double2* __restrict__ F, double s,
                                          const double2* __restrict__ U = nullptr) {
  if (!(fl & FL_PRE)) hph_op<RB, B, 0, false, SC, REAL>(a, W, F, s, U);
  else if (!(fl & FL_REG)) hph_op<RB, B, 1, false, SC, REAL>(a, W, F, s, U);
  else if (fl & FL_LOWF) hph_op<RB, B, 2, true, SC, REAL>(a, W, F, s, U);
  else hph_op<RB, B, 2, false, SC, REAL>(a, W, F, s, U);
}

// Sub-op kinds a build of the straight-line phases handles.
enum : int { HPK_H = 1, HPK_R = 2, HPK_ANY = 3 };

// sub-op I of K (register bit I), then the rest.  KINDS: HPK_H (Hadamard-
// pattern sub-ops only), HPK_R (real 2x2 only) or HPK_ANY.
template <int RB, int K, int I, int KINDS>
__device__ __forceinline__ void hph_run(double2 (&a)[1 << RB], const uint4* __restrict__ SUB,
                                        const double2* __restrict__ DATA,
                                        const double2* __restrict__ slots, uint32_t tid, double s,
                                        bool sc) {
  if constexpr (I < K) {
    const uint4 o0 = SUB[2 * I];
    const uint32_t fl = (o0.y >> 8) & 0xffu;
    const double2* T = DATA + o0.z + 4;
    double2 W = make_double2(1.0, 0.0);
    if (fl & FL_PRE) {
      W = slots[o0.y >> 16];
      if (fl & FL_THR) {
        W = cmul_f(W, cmul_f(T[tid & 31u], T[32 + (tid >> 5)]));
        T += 40;
      }
    }
    if constexpr (KINDS == HPK_R) {
      hph_flags<RB, I, false, true>(a, fl, W, T, s, DATA + o0.z);
    } else {
      if (KINDS == HPK_ANY && (o0.x & 0xffu) == OP_U1R) {  // the phase's scale belongs to its H ops
        if constexpr (KINDS == HPK_ANY) hph_flags<RB, I, false, true>(a, fl, W, T, s, DATA + o0.z);
      } else if (I == K - 1 && sc) {
        W = make_double2(W.x * s, W.y * s);
        hph_flags<RB, I, true>(a, fl, W, T, s);
      } else {
        hph_flags<RB, I, false>(a, fl, W, T, s);
      }
    }
    hph_run<RB, K, I + 1, KINDS>(a, SUB, DATA, slots, tid, s, sc);
  }
}

// An OP_HPHASE marker (hdr) and its sub-ops at SUB (two uint4 per op).
template <int RB, int KINDS = HPK_ANY>
__device__ __forceinline__ void h_phase(const uint4 hdr, const uint4* __restrict__ SUB,
                                        double2 (&a)[1 << RB], const double2* __restrict__ DATA,
                                        const double2* __restrict__ slots, uint32_t tid) {
  const uint32_t K = (hdr.x >> 16) & 0xffu;
  const bool sc = ((hdr.y >> 8) & HPH_SCALE) != 0u;
  const double s = sc ? DATA[hdr.z].x : 1.0;
  switch (K) {
    case 1: hph_run<RB, 1, 0, KINDS>(a, SUB, DATA, slots, tid, s, sc); break;
    case 2: if constexpr (RB >= 2) hph_run<RB, 2, 0, KINDS>(a, SUB, DATA, slots, tid, s, sc); break;
    case 3: if constexpr (RB >= 3) hph_run<RB, 3, 0, KINDS>(a, SUB, DATA, slots, tid, s, sc); break;
    case 4: if constexpr (RB >= 4) hph_run<RB, 4, 0, KINDS>(a, SUB, DATA, slots, tid, s, sc); break;
    default: break;
  }
}

// The interpreter for SWF_UONLY programs: one-qubit ops (general, real, X)
// with register, thread or non-local controls and no flush.
template <int RB>
__device__ __forceinline__ void exec_u(const uint4 o0, const uint4 o1, double2 (&a)[1 << RB],
                                       const double2* __restrict__ DATA, uint32_t tid,
                                       uint64_t base) {
  const uint32_t type = o0.x & 0xffu, b0 = (o0.x >> 8) & 0xffu;
  const uint32_t creg = o0.x >> 24, ctl = o0.y & 0xffu;
  const uint64_t cnl = ((uint64_t)o1.y << 32) | o1.x;
  if ((base & cnl) != cnl) return;
  if ((tid & ctl) != ctl) return;
  const double2* D = DATA + o0.z;
  const double2 W = make_double2(1.0, 0.0);
  const double2* F = nullptr;
  if (type == OP_U1) {
    DQ_SW_U1(0, 0)
  } else if (type == OP_U1R) {
    DQ_SW_U1(1, 0)
  } else {
    DQ_SW_U1(3, 0)
  }
}

template <int RB>
__device__ __forceinline__ void exec_op(const uint4 o0, const uint4 o1, double2 (&a)[1 << RB],
                                        const double2* __restrict__ DATA,
                                        const double2* __restrict__ slots, uint32_t tid,
                                        uint64_t base) {
  const uint32_t type = o0.x & 0xffu, b0 = (o0.x >> 8) & 0xffu, b1 = (o0.x >> 16) & 0xffu;
  const uint32_t creg = o0.x >> 24, ctl = o0.y & 0xffu, flags = (o0.y >> 8) & 0xffu;
  const uint32_t slot = o0.y >> 16;
  const uint64_t cnl = ((uint64_t)o1.y << 32) | o1.x;
  if ((base & cnl) != cnl) return;
  if ((tid & ctl) != ctl) return;
  const double2* D = DATA + o0.z;
  // flush factors (FLUSH ops and pre-flushed one-qubit ops)
  double2 W = make_double2(1.0, 0.0);
  const double2* F = nullptr;
  const bool is_u1 = type == OP_U1 || type == OP_U1R || type == OP_U1H || type == OP_U1X;
  if ((flags & FL_PRE) || type == OP_FLUSH_R || type == OP_FLUSH_T || type == OP_GPHASE) {
    W = slots[slot];
    const double2* T = is_u1 ? D + 4 : D;
    if (flags & FL_THR) {
      W = cmul_f(W, cmul_f(T[tid & 31u], T[32 + (tid >> 5)]));
      T += 40;
    }
    if (flags & FL_REG) F = T;
  }
  switch (type) {
    case OP_U1:
      if (!(flags & FL_PRE)) { DQ_SW_U1(0, 0) } else if (F) { DQ_SW_U1(0, 2) } else { DQ_SW_U1(0, 1) }
      break;
    case OP_U1R:
      if (!(flags & FL_PRE)) { DQ_SW_U1(1, 0) } else if (F) { DQ_SW_U1(1, 2) } else { DQ_SW_U1(1, 1) }
      break;
    case OP_U1H:
      if (!(flags & FL_PRE)) { DQ_SW_U1(2, 0) } else if (F) { DQ_SW_U1(2, 2) } else { DQ_SW_U1(2, 1) }
      break;
    case OP_U1X:
      if (!(flags & FL_PRE)) { DQ_SW_U1(3, 0) } else if (F) { DQ_SW_U1(3, 2) } else { DQ_SW_U1(3, 1) }
      break;
    case OP_U2: u2_dispatch<RB>(a, b0, b1, creg, D); break;
    case OP_FLUSH_R: DQ_SW_CASES1(flush_reg, a, W, F); break;
    case OP_FLUSH_T:
      if (!((tid >> b0) & 1u)) break;
      if (F) {
#pragma unroll
        for (int j = 0; j < (1 << RB); ++j) a[j] = cmul_f(a[j], cmul_f(W, F[j]));
      } else {
#pragma unroll
        for (int j = 0; j < (1 << RB); ++j) a[j] = cmul_f(a[j], W);
      }
      break;
    case OP_GPHASE:
#pragma unroll
      for (int j = 0; j < (1 << RB); ++j) a[j] = cmul_f(a[j], W);
      break;
    case OP_SCALE: {
      const double f = D[0].x;
#pragma unroll
      for (int j = 0; j < (1 << RB); ++j) a[j] = make_double2(a[j].x * f, a[j].y * f);
      break;
    }
    default: break;
  }
}

// The per-CTA tile loop of a sweep: tiles first_tile, first_tile +
// tile_step, ... (< ntiles) of the program at `prog` (shared or global
// memory), with S tile buffers at `bufs` and the per-tile slot factors at
// `slots` (shared memory).  Every thread of the CTA calls it; no copy is in
// flight on return.  S tile buffers form a cp.async pipeline with S - 1
// tiles prefetched while the current one is computed.
// RUNB: the program's run_bits (5 or 3), fixed at compile time.  HONLY: the
// program's phases are all H phases (SWF_HONLY), so the generic op
// interpreter is left out of the build.  FORM: FORM_H for SWF_HONLY programs
// (no op interpreter), FORM_U for SWF_UONLY programs (the one-qubit part of
// it), FORM_ALL otherwise.
template <int TB, int RB, int S, int RUNB, int FORM = FORM_ALL>
__device__ __forceinline__ void sweep_tiles(double2* __restrict__ state, const uint8_t* prog,
                                            uint32_t ntiles, long long synth, double2* bufs,
                                            double2* slots, uint32_t first_tile, uint32_t tile_step) {
  constexpr int kSwThreads = 1 << TB;
  constexpr int kSwTB = TB;
  constexpr int M = kSwTB + RB;
  constexpr int T = 1 << M;
  constexpr int R = 1 << RB;
  constexpr int NI = 1 << (M - kSwTB);  // 32-element chunks per warp
  constexpr uint32_t NW = 1u << (TB - 5);  // warps
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const SwHeader* H = reinterpret_cast<const SwHeader*>(prog);
  const SwPhase* PH = reinterpret_cast<const SwPhase*>(prog + H->off_phase);
  const SwOp* OPS = reinterpret_cast<const SwOp*>(prog + H->off_op);
  const SwSlot* SL = reinterpret_cast<const SwSlot*>(prog + H->off_slot);
  const SwSlotEnt* SE = reinterpret_cast<const SwSlotEnt*>(prog + H->off_slotent);
  const double2* DATA = reinterpret_cast<const double2*>(prog + H->off_data);
  const uint64_t* RUNOFF = reinterpret_cast<const uint64_t*>(prog + H->off_runoff);
  const uint32_t* RUNSWZ = reinterpret_cast<const uint32_t*>(prog + H->off_runswz);
  const uint32_t nph = H->nphase, nslots = H->nslots;
  const SwGStore* GS =
      (H->off_gstore && nph) ? reinterpret_cast<const SwGStore*>(prog + H->off_gstore) : nullptr;
  // element e = 32 c + lane of a tile (c: the warp's chunk) lies in run
  // e >> run_bits at offset e & (2^run_bits - 1)
  constexpr uint32_t run_bits = RUNB, cshift = 5u - RUNB;
  const uint32_t lane_run = lane >> run_bits, lane_off = lane & ((1u << run_bits) - 1u);
  const uint32_t swl = swz(lane_off);  // the offset's part of the swizzled index

  auto tile_base = [&](uint32_t t) {
    uint64_t b = t;
#pragma unroll
    for (int k = 0; k < M; ++k) b = insert_zero(b, H->local_pos[k]);
    return b;
  };
  // Tile bases advance by the grid stride without re-depositing: with the
  // local positions filled with ones a carry runs across them, so
  // deposit(t + g) = ((deposit(t) | lmask) + deposit(g)) & ~lmask.
  uint64_t lmask = 0;
#pragma unroll
  for (int k = 0; k < M; ++k) lmask |= 1ULL << H->local_pos[k];
  const uint64_t bstride = tile_base(tile_step);
  auto advance = [&](uint64_t b) { return ((b | lmask) + bstride) & ~lmask; };
  // chunk warp + NW i (32 elements): all of a tile's runs; one commit
  // group per call (empty past the last tile, so the group count is
  // uniform).  synth >= 0: the state is the basis vector |synth> not yet
  // written to memory, so the tile is generated instead of read.  A
  // generated tile that does not hold the basis index is zero and stays
  // zero through every (linear) op of the sweep: it is neither generated
  // nor computed, only written as zeros.
  const uint64_t synth_base = synth >= 0 ? ((uint64_t)synth & ~lmask) : ~0ULL;
  auto zero_tile = [&](uint64_t b) { return synth >= 0 && b != synth_base; };
  auto load_tile = [&](uint32_t t, uint64_t b, double2* dst) {
    if (t < ntiles && !zero_tile(b)) {
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const uint32_t r = ((warp + (uint32_t)i * NW) << cshift) + lane_run;
        const uint64_t g = b + RUNOFF[r] + lane_off;
        double2* d = &dst[RUNSWZ[r] ^ swl ^ H->tile_xload];
        if (synth >= 0)
          *d = make_double2(g == (uint64_t)synth ? 1.0 : 0.0, 0.0);
        else
          cp_async16(d, state + g);
      }
    }
    cp_async_commit();
  };

  uint32_t tile = first_tile;
  uint64_t base = tile_base(tile);  // this iteration's tile
  uint64_t bpre = base;             // the newest prefetched tile
#pragma unroll
  for (int k = 0; k < S - 1; ++k) {
    load_tile(tile + (uint32_t)k * tile_step, bpre, bufs + k * T);
    bpre = advance(bpre);
  }
  for (uint32_t it = 0; tile < ntiles; ++it, tile += tile_step) {
    double2* cur = bufs + (it % S) * T;
    // tile it + S - 1 goes into the buffer that tile it - 1 used (stored and
    // released by the barrier that ended the previous iteration)
    load_tile(tile + (uint32_t)(S - 1) * tile_step, bpre, bufs + ((it + S - 1) % S) * T);
    bpre = advance(bpre);
    if (zero_tile(base)) {  // uniform over the CTA
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const uint32_t r = ((warp + (uint32_t)i * NW) << cshift) + lane_run;
        state[base + RUNOFF[r] + lane_off] = make_double2(0.0, 0.0);
      }
      base = advance(base);
      continue;
    }
    // per-tile phase factors: up to 16 slots per warp take an 8-lane group
    // each (lane products over every 8th entry, then a three-round butterfly
    // over the group); more slots take one thread each
    if (nslots <= 16 * NW) {
      const uint32_t gl = lane & 7u, grp = lane >> 3;
      for (uint32_t s0 = warp * 4u; s0 < nslots; s0 += NW * 4u) {
        const uint32_t s = s0 + grp;
        double2 w = make_double2(1.0, 0.0);
        if (s < nslots) {
          const uint32_t c = SL[s].count, st = SL[s].start;
          for (uint32_t e = gl; e < c; e += 8u) {
            const SwSlotEnt& E = SE[st + e];
            if ((base & E.mask) == E.mask) w = cmul_f(w, E.w);
          }
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
          const double2 q = make_double2(__shfl_xor_sync(0xffffffffu, w.x, o),
                                         __shfl_xor_sync(0xffffffffu, w.y, o));
          w = cmul_f(w, q);
        }
        if (gl == 0 && s < nslots) slots[s] = cmul_f(SL[s].w0, w);
      }
    } else {
      for (uint32_t s = tid; s < nslots; s += kSwThreads) {
        double2 w = SL[s].w0;
        const uint32_t c = SL[s].count, st = SL[s].start;
        for (uint32_t e = 0; e < c; ++e) {
          const SwSlotEnt& E = SE[st + e];
          if ((base & E.mask) == E.mask) w = cmul_f(w, E.w);
        }
        slots[s] = w;
      }
    }
    cp_async_wait<S - 1>();  // this tile's group is complete; S - 1 newer may be pending
    __syncthreads();

    for (uint32_t p = 0; p < nph; ++p) {
      const SwPhase& P = PH[p];
      const uint32_t pt = P.lanesw[lane] ^ P.warpsw[warp];
      const uint32_t ptl = pt ^ P.xload;
      uint32_t V[RB];
#pragma unroll
      for (int b = 0; b < RB; ++b) V[b] = P.V[b];
      double2 a[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        uint32_t x = ptl;
#pragma unroll
        for (int b = 0; b < RB; ++b)
          if ((j >> b) & 1) x ^= V[b];
        a[j] = cur[x];
      }
      const uint32_t ob = P.op_begin, oe = P.op_end;
      const uint4* OP4 = reinterpret_cast<const uint4*>(OPS);
      uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
      if (ob < oe) {
        c0 = OP4[2 * ob];
        c1 = OP4[2 * ob + 1];
      }
      if constexpr (FORM == FORM_H) {
        h_phase<RB, HPK_H>(c0, OP4 + 2 * ob + 2, a, DATA, slots, tid);
      } else if constexpr (FORM == FORM_R) {
        h_phase<RB, HPK_R>(c0, OP4 + 2 * ob + 2, a, DATA, slots, tid);
      } else if constexpr (FORM == FORM_U) {
        for (uint32_t o = ob; o < oe; ++o) {
          uint4 n0 = c0, n1 = c1;
          if (o + 1 < oe) {
            n0 = OP4[2 * o + 2];
            n1 = OP4[2 * o + 3];
          }
          exec_u<RB>(c0, c1, a, DATA, tid, base);
          c0 = n0;
          c1 = n1;
        }
      } else if (ob < oe && (c0.x & 0xffu) == OP_HPHASE) {
        h_phase<RB>(c0, OP4 + 2 * ob + 2, a, DATA, slots, tid);
      } else {
        for (uint32_t o = ob; o < oe; ++o) {
          uint4 n0 = c0, n1 = c1;
          if (o + 1 < oe) {  // next descriptor in flight while this op runs
            n0 = OP4[2 * o + 2];
            n1 = OP4[2 * o + 3];
          }
          exec_op<RB>(c0, c1, a, DATA, slots, tid, base);
          c0 = n0;
          c1 = n1;
        }
      }
      if (GS && p + 1 == nph) {
        // the last phase writes its amplitudes straight to the state; the
        // barrier that ends the tile orders these reads of cur before the
        // next tile's load into it
        const uint64_t gt = base + GS->glane[lane] + GS->gwarp[warp];
#pragma unroll
        for (int j = 0; j < R; ++j) {
          uint64_t g = gt;
#pragma unroll
          for (int b = 0; b < RB; ++b)
            if ((j >> b) & 1) g += GS->gV[b];
          state[g] = a[j];
        }
        continue;
      }
      const uint32_t pt2 = opaque(pt);
#pragma unroll
      for (int b = 0; b < RB; ++b) V[b] = opaque(V[b]);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        uint32_t x = pt2;
#pragma unroll
        for (int b = 0; b < RB; ++b)
          if ((j >> b) & 1) x ^= V[b];
        cur[x] = a[j];
      }
      __syncthreads();
    }

    if (!GS) {
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const uint32_t r = ((warp + (uint32_t)i * NW) << cshift) + lane_run;
        state[base + RUNOFF[r] + lane_off] = cur[RUNSWZ[r] ^ swl];
      }
    }
    base = advance(base);
    __syncthreads();
  }
  cp_async_wait<0>();
}

}  // namespace
}  // namespace dq
