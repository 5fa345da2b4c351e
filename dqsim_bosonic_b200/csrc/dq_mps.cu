// dq_mps.cu — matrix-product-state backend on the device.
//
// Restates the MPS simulator of the reference (src/monolithic/mps/simulator.rs):
// one rank-3 tensor A_k[l][s][r] per qubit k, bond dimensions dims[0..n]
// (dims[0] = dims[n] = 1), single-qubit gates contracted into one tensor
// (apply_1q, :99-113), two-qubit gates as a chain of adjacent steps (apply_2q,
// :115-135) whose every step contracts the two tensors with the 4x4 gate into
// theta (2L x 2R), takes its SVD, truncates and splits it again
// (apply_adjacent_2q, :137-236), measurement by p1 / draw / projection
// (measure, project_qubit, :259-291) and reset = measure + X.
//
// B200 design: a batch of B independent MPS (one per shot; B = 1 for
// `simulate`) lives in HBM with padded tensors (capacity `cap` per bond) and
// per-replica bond dimensions on the device.  Every launch runs one program
// operation, or a run of operations on pairwise disjoint sites (they commute
// exactly; blockIdx.y selects the operation), over the whole batch, so the host
// never reads a bond dimension while the program runs:
//   k_mps_1q       the 2x2 contraction of one site (exact num-complex order)
//   k_mps_2q       FUSED adjacent step, one CTA per replica: theta build,
//                  one-sided (Hestenes) Jacobi SVD in shared memory (global
//                  memory above capacity 32), descending sort, truncation with
//                  the reference's keep / renormalisation rule, split into the
//                  two new site tensors, new bond dimension
//   k_mps_2q_warp  the same step with one warp per replica (large batches of
//                  bonds <= 16)
//   k_mps_measure  p1 by a transfer-matrix contraction over the chain
//   (and _warp)    (O(n chi^3) instead of the reference's 2^n statevector),
//                  the replica's ChaCha8 draw, projection, reset flip, cbit
//   k_mps_expand   to_statevector (:238-257) as a left-to-right contraction,
//                  one launch per site, same summation order as the reference
// Conditions are evaluated per replica on the device.  When a truncation
// keeps more singular values than the capacity, the kernel flags it and the
// host re-runs the (deterministic) program with a larger capacity.
//
// The SVD differs from nalgebra's (Golub-Kahan) in the gauge of U and V, so
// site tensors are not bit-identical to the reference; everything a caller
// can observe (statevector, probabilities, outcomes) is gauge-invariant and
// held to a tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "dq_common.cuh"
#include "dq_gates.hpp"
#include "dq_handle.cuh"
#include "dq_rng.cuh"

namespace dq {
namespace {

enum MpsOpKind : int32_t { M_1Q = 0, M_2Q = 1, M_MEAS = 2, M_RESET = 3, M_FAIL = 4 };

struct MpsOp {
  int32_t kind;
  uint32_t q;            // site (M_2Q: left site of the bond q, q+1)
  int32_t cbit;          // M_MEAS: classical bit written
  uint32_t cond_first;   // condition chain (all must hold)
  uint32_t cond_count;
  int32_t inst;          // instruction index (error reports)
  double2 u[16];         // M_1Q: 2x2 row-major in u[0..3]; M_2Q: 4x4 row-major
};

// Device view of a batch.
struct MpsView {
  double2* t;            // site k of replica b at t + (k * batch + b) * site_elems
  uint32_t* dims;        // batch x (n + 1)
  const uint32_t* key;   // batch x 8 ChaCha8 key words
  unsigned long long* ctr;  // batch: draws consumed
  int32_t* cbits;        // batch x ncb
  const dq_cond* conds;
  double2* scratch;      // batch x scratch_elems (global fallback of the SVD work area)
  int* flags;            // [0] status, [1] first failing instruction, [2] capacity needed
  unsigned long long* svd_calls;
  const MpsOp* ops;      // the program's operations; a launch runs ops[first + blockIdx.y]
  uint64_t site_elems;   // cap * 2 * cap
  uint64_t scratch_elems;
  uint32_t n, batch, cap, ncb;
  uint32_t slots;        // scratch slots per replica (two-qubit steps per launch)
};

enum : int { MF_OK = 0, MF_UNSUPPORTED = 1, MF_CAPACITY = 2 };

constexpr int kMpsThreads = 256;
constexpr int kMaxSweeps = 60;

__device__ __forceinline__ double2* site(const MpsView& v, uint32_t k, uint32_t b) {
  return v.t + ((uint64_t)k * v.batch + b) * v.site_elems;
}

__device__ __forceinline__ bool cond_ok(const MpsView& v, const MpsOp& op, uint32_t b) {
  const int32_t* cb = v.cbits + (uint64_t)b * v.ncb;
  for (uint32_t c = 0; c < op.cond_count; ++c) {
    const dq_cond cd = v.conds[op.cond_first + c];
    uint64_t actual = 0;
    for (uint64_t i = 0; i < cd.creg_size; ++i) {
      const uint64_t idx = cd.creg_base + i;
      const uint64_t bit = (idx < v.ncb && cb[idx] > 0) ? (uint64_t)cb[idx] : 0;
      actual |= bit << i;
    }
    if (actual != cd.creg_value) return false;
  }
  return true;
}

// new[l][o][r] = sum_i u[o][i] old[l][i][r], accumulated from zero in the
// reference's order (apply_1q, simulator.rs:99-113).
__device__ void site_1q(double2* a, uint32_t L, uint32_t R, uint32_t cap, const double2* u) {
  const double2 zero = make_double2(0.0, 0.0);
  for (uint32_t t = threadIdx.x; t < L * R; t += blockDim.x) {
    const uint32_t l = t / R, r = t - (t / R) * R;
    double2* p0 = a + (uint64_t)(l * 2) * cap + r;
    double2* p1 = p0 + cap;
    const double2 a0 = *p0, a1 = *p1;
    *p0 = cadd_x(cadd_x(zero, cmul_x(u[0], a0)), cmul_x(u[1], a1));
    *p1 = cadd_x(cadd_x(zero, cmul_x(u[2], a0)), cmul_x(u[3], a1));
  }
}

__global__ void __launch_bounds__(kMpsThreads) k_mps_reset(MpsView v) {
  const uint32_t b = blockIdx.x;
  for (uint32_t k = 0; k < v.n; ++k) {
    double2* a = site(v, k, b);
    if (threadIdx.x == 0) a[0] = make_double2(1.0, 0.0);   // |0>: A[0][0][0] = 1
    if (threadIdx.x == 1) a[v.cap] = make_double2(0.0, 0.0);  // A[0][1][0] = 0
  }
  for (uint32_t k = threadIdx.x; k <= v.n; k += blockDim.x) v.dims[(uint64_t)b * (v.n + 1) + k] = 1;
  for (uint32_t c = threadIdx.x; c < v.ncb; c += blockDim.x) v.cbits[(uint64_t)b * v.ncb + c] = -1;
  if (threadIdx.x == 0) v.ctr[b] = 0;
}

__global__ void __launch_bounds__(kMpsThreads) k_mps_1q(MpsView v, uint32_t first) {
  const MpsOp& op = v.ops[first + blockIdx.y];
  const uint32_t b = blockIdx.x;
  if (!cond_ok(v, op, b)) return;
  const uint32_t* dm = v.dims + (uint64_t)b * (v.n + 1);
  site_1q(site(v, op.q, b), dm[op.q], dm[op.q + 1], v.cap, op.u);
}

__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Rotation of one column pair (p, q) with Gram entries alpha = |a_p|^2,
// beta = |a_q|^2, gamma = a_p^H a_q = |gamma| e^{i phi}: false when the pair
// is orthogonal to within tol.  Otherwise
//   a_p' = c a_p - s e^{-i phi} a_q,   a_q' = s e^{i phi} a_p + c a_q
// with t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = (beta - alpha) /
// (2 |gamma|), c = 1 / sqrt(1 + t^2), s = c t, which zeroes a_p'^H a_q'.  The
// reciprocal square roots keep the dependent chain at four special-function
// operations.
//
// A pair of negligible columns (both |a|^2 <= neg = (rows eps)^2 |theta|_F^2,
// at the rounding level of theta) is left alone: their mutual directions carry
// no information and rotating them again and again only delays convergence of
// a rank-deficient theta.  A negligible column is still rotated against every
// significant one, so it ends up orthogonal to the significant subspace.  When
// the threshold keeps such a column (a threshold at or below the rounding
// level), the split writes it as zeros: its vector is not orthogonal to the
// other negligible ones, and dividing by its sigma would put O(1) entries
// into the left tensor for a contribution of order eps |theta|.  The bond
// dimension is the reference's either way.
__device__ __forceinline__ bool jacobi_rotation(double al, double be, double gr, double gi, double tol,
                                                double neg, double& c, double& s, double& ex, double& ey) {
  const double g2 = gr * gr + gi * gi;
  if (!(g2 > 0.0)) return false;
  if (al <= neg && be <= neg) return false;
  const double nab = sqrt(al) * sqrt(be);
  const double inv = rsqrt(g2);
  if (!(g2 * inv > tol * nab)) return false;
  const double zeta = 0.5 * (be - al) * inv;
  const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
  c = rsqrt(1.0 + t * t);
  s = c * t;
  ex = gr * inv;
  ey = gi * inv;
  return true;
}

// Work area (double2 elements) of the fused step at capacity cap, in shared
// memory when it fits: G (rows x cols <= 4 cap^2) + sigma (cols doubles) +
// perm (cols u32).  The measurement kernel uses it for three cap x cap
// transfer matrices.
__host__ __device__ inline uint64_t svd_work_elems(uint32_t cap) {
  const uint64_t c = 2ull * cap;
  return c * c + c + (c + 1) / 2;
}
// theta copy (row-major 2L x 2R <= 4 cap^2), always in global memory
__host__ __device__ inline uint64_t theta_elems(uint32_t cap) { return 4ull * cap * cap; }

// Fused adjacent two-qubit step on bond (q, q+1) of every replica.
//   theta[(l*2+o0)][(o1*R+r)] = sum_in u[o][in] sum_k A[l][in0][k] B[k][in1][r]
// (apply_adjacent_2q, simulator.rs:148-171; same accumulation order).  The
// SVD is one-sided Jacobi on G = theta (2R <= 2L) or G = theta^H (2R > 2L):
// column pairs of a round-robin tournament (each round cols/2 disjoint pairs,
// one warp per pair) are rotated until every pair is orthogonal to within
// rows * eps, leaving G = W V^H with orthogonal columns W_j = sigma_j u_j.
// V is never formed: with U = W / sigma the split tensors are
//   2R <= 2L:  left = U,                       right = scale * U^H theta
//   2R >  2L:  left = theta W / sigma^2,       right = scale * W^H
// read from a copy of theta (global memory, L2-resident).
__global__ void __launch_bounds__(1024) k_mps_2q(MpsView v, uint32_t first, uint32_t max_keep, double thr,
                                                 int use_smem) {
  const MpsOp& op = v.ops[first + blockIdx.y];
  extern __shared__ double2 smem[];
  __shared__ int s_rot;
  __shared__ uint32_t s_keep;
  __shared__ double s_scale;
  __shared__ double s_part[32];
  __shared__ double s_n2;
  const uint32_t b = blockIdx.x;
  if (!cond_ok(v, op, b)) return;
  uint32_t* dm = v.dims + (uint64_t)b * (v.n + 1);
  const uint32_t q = op.q, cap = v.cap;
  const uint32_t L = dm[q], M = dm[q + 1], R = dm[q + 2];
  const bool tr = R > L;
  const uint32_t rows = tr ? 2 * R : 2 * L, cols = tr ? 2 * L : 2 * R;
  const uint32_t tw = 2 * R;   // theta row length
  double2* TH = v.scratch + ((uint64_t)b * v.slots + blockIdx.y) * v.scratch_elems;
  double2* G = use_smem ? smem : TH + theta_elems(cap);
  double* sig = reinterpret_cast<double*>(G + (uint64_t)rows * cols);
  uint32_t* perm = reinterpret_cast<uint32_t*>(sig + cols);
  double2* A = site(v, q, b);
  double2* B = site(v, q + 1, b);
  const double2 zero = make_double2(0.0, 0.0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;

  // ---- theta -> TH (row-major) and G (column-major) ---------------------------
  double n2loc = 0.0;  // |theta|_F^2, for the negligible-pair test
  for (uint32_t t = tid; t < L * R; t += blockDim.x) {
    const uint32_t l = t / R, r = t - (t / R) * R;
    double2 in[4];
    for (int i0 = 0; i0 < 2; ++i0)
      for (int i1 = 0; i1 < 2; ++i1) {
        double2 acc = zero;
        const double2* ar = A + (uint64_t)(l * 2 + i0) * cap;
        for (uint32_t k = 0; k < M; ++k)
          acc = cadd_x(acc, cmul_x(ar[k], B[(uint64_t)(k * 2 + i1) * cap + r]));
        in[i0 * 2 + i1] = acc;
      }
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1) {
        const int o = o0 * 2 + o1;
        double2 acc = zero;
        for (int i = 0; i < 4; ++i) acc = cadd_x(acc, cmul_x(op.u[o * 4 + i], in[i]));
        const uint32_t row = l * 2 + o0, col = o1 * R + r;
        TH[(uint64_t)row * tw + col] = acc;
        n2loc += acc.x * acc.x + acc.y * acc.y;
        if (!tr) G[(uint64_t)col * rows + row] = acc;
        else G[(uint64_t)row * rows + col] = make_double2(acc.x, -acc.y);
      }
  }
  n2loc = warp_sum(n2loc);
  if (lane == 0) s_part[warp] = n2loc;
  if (tid == 0) s_rot = 0;
  __syncthreads();
  if (tid == 0) {
    double n2 = 0.0;
    for (int w = 0; w < nw; ++w) n2 += s_part[w];
    s_n2 = n2;
  }
  __syncthreads();

  // ---- one-sided Jacobi --------------------------------------------------------
  const double tol = (double)rows * DBL_EPSILON;
  const double neg = tol * tol * s_n2;
  const uint32_t np = cols / 2;
  // more pairs than warps: two lane groups of 16 lanes, one pair each, so that
  // two of a warp's pairs run side by side (narrower groups would leave each
  // lane a long serial run of loads)
  const uint32_t ppw = (np + nw - 1) / nw;
  const uint32_t lpp = ppw > 1 ? 16u : 32u;
  const uint32_t gpw = 32 / lpp, g = (uint32_t)lane / lpp, h = (uint32_t)lane % lpp;
  for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
    for (uint32_t rd = 0; rd + 1 < cols; ++rd) {
      for (uint32_t base = warp * gpw; base < np; base += nw * gpw) {
        const uint32_t pi = base + g;
        const bool active = pi < np;
        uint32_t p = 0, qq = 0;
        if (active) {
          if (pi == 0) {
            p = rd;
            qq = cols - 1;
          } else {
            p = (rd + pi) % (cols - 1);
            qq = (rd + (cols - 1) - pi) % (cols - 1);
          }
        }
        double2* gp = G + (uint64_t)p * rows;
        double2* gq = G + (uint64_t)qq * rows;
        double al = 0.0, be = 0.0, gr = 0.0, gi = 0.0;
        if (active)
          for (uint32_t i = h; i < rows; i += lpp) {
            const double2 x = gp[i], y = gq[i];
            al += x.x * x.x + x.y * x.y;
            be += y.x * y.x + y.y * y.y;
            gr += x.x * y.x + x.y * y.y;
            gi += x.x * y.y - x.y * y.x;
          }
        for (uint32_t o = lpp / 2; o >= 1; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          gr += __shfl_xor_sync(0xffffffffu, gr, o);
          gi += __shfl_xor_sync(0xffffffffu, gi, o);
        }
        double c, s, ex, ey;
        if (active && jacobi_rotation(al, be, gr, gi, tol, neg, c, s, ex, ey)) {
          if (h == 0) s_rot = 1;
          for (uint32_t i = h; i < rows; i += lpp) {
            const double2 x = gp[i], y = gq[i];
            gp[i] = make_double2(c * x.x - s * (ex * y.x + ey * y.y), c * x.y - s * (ex * y.y - ey * y.x));
            gq[i] = make_double2(s * (ex * x.x - ey * x.y) + c * y.x, s * (ex * x.y + ey * x.x) + c * y.y);
          }
        }
      }
      __syncthreads();
    }
    const int rot = s_rot;
    __syncthreads();
    if (!rot) break;
    if (tid == 0) s_rot = 0;
    __syncthreads();
  }

  // ---- singular values, descending order (ties by column index) ---------------
  for (uint32_t j = warp; j < cols; j += nw) {
    const double2* g = G + (uint64_t)j * rows;
    double s = 0.0;
    for (uint32_t i = lane; i < rows; i += 32) s += g[i].x * g[i].x + g[i].y * g[i].y;
    s = warp_sum(s);
    if (lane == 0) sig[j] = sqrt(s);
  }
  __syncthreads();
  for (uint32_t j = tid; j < cols; j += blockDim.x) {
    uint32_t rank = 0;
    const double sj = sig[j];
    for (uint32_t i = 0; i < cols; ++i) rank += (sig[i] > sj || (sig[i] == sj && i < j)) ? 1u : 0u;
    perm[rank] = j;
  }
  __syncthreads();

  // ---- truncation (simulator.rs:186-218) ----------------------------------------
  if (tid == 0) {
    uint32_t keep = 0;
    for (uint32_t k = 0; k < cols; ++k) keep += sig[perm[k]] > thr ? 1u : 0u;
    keep = keep > 1u ? keep : 1u;
    if (max_keep) keep = keep < max_keep ? keep : max_keep;
    double kept = 0.0, total = 0.0, disc = 0.0;
    for (uint32_t k = 0; k < keep; ++k) kept += sig[perm[k]] * sig[perm[k]];
    for (uint32_t k = 0; k < cols; ++k) total += sig[perm[k]] * sig[perm[k]];
    for (uint32_t k = keep; k < cols; ++k) disc += sig[perm[k]] * sig[perm[k]];
    kept = fmax(sqrt(kept), 1e-15);
    total = sqrt(total);
    s_scale = disc > 0.0 ? total / kept : 1.0;
    s_keep = keep;
    if (keep > cap) {
      atomicMax(&v.flags[2], (int)keep);
      atomicMax(&v.flags[0], MF_CAPACITY);
    } else {
      atomicAdd(v.svd_calls, 1ull);
    }
  }
  __syncthreads();
  const uint32_t keep = s_keep;
  if (keep > cap) return;
  const double scale = s_scale;

  // ---- split ----------------------------------------------------------------------
  for (uint32_t t = tid; t < L * 2 * keep; t += blockDim.x) {
    const uint32_t row = t / keep, k = t - (t / keep) * keep;   // row = l*2 + s
    const uint32_t j = perm[k];
    const double sj = sig[j];
    double2 val = zero;
    if (sj > 0.0 && sj * sj > neg) {  // a kept column at the rounding level of theta is left zero
      if (!tr) {
        const double2 g = G[(uint64_t)j * rows + row];
        val = make_double2(g.x / sj, g.y / sj);
      } else {
        // (theta W_j)[row] / sigma_j^2
        const double2* th = TH + (uint64_t)row * tw;
        const double2* w = G + (uint64_t)j * rows;
        double re = 0.0, im = 0.0;
        for (uint32_t c2 = 0; c2 < tw; ++c2) {
          const double2 a = th[c2], x = w[c2];
          re += a.x * x.x - a.y * x.y;
          im += a.x * x.y + a.y * x.x;
        }
        const double s2 = sj * sj;
        val = make_double2(re / s2, im / s2);
      }
    }
    A[(uint64_t)row * cap + k] = val;
  }
  for (uint32_t t = tid; t < keep * 2 * R; t += blockDim.x) {
    const uint32_t k = t / (2 * R), col = t - (t / (2 * R)) * (2 * R);  // col = s*R + r
    const uint32_t s = col / R, r = col - (col / R) * R;
    const uint32_t j = perm[k];
    const double sj = sig[j];
    double2 val = zero;
    if (sj > 0.0 && sj * sj > neg) {  // a kept column at the rounding level of theta is left zero
      if (tr) {
        const double2 g = G[(uint64_t)j * rows + col];
        val = make_double2(scale * g.x, -scale * g.y);
      } else {
        // scale * (U_j^H theta)[col], U_j = W_j / sigma_j
        const double2* w = G + (uint64_t)j * rows;
        double re = 0.0, im = 0.0;
        for (uint32_t r2 = 0; r2 < rows; ++r2) {
          const double2 x = w[r2], a = TH[(uint64_t)r2 * tw + col];
          re += x.x * a.x + x.y * a.y;
          im += x.x * a.y - x.y * a.x;
        }
        const double f = scale / sj;
        val = make_double2(f * re, f * im);
      }
    }
    B[(uint64_t)(k * 2 + s) * cap + r] = val;
  }
  if (tid == 0) dm[q + 1] = keep;
}

// Batched form of k_mps_2q for capacity <= 16 (theta at most 32 x 32): two
// warps (64 lanes) per replica, kRepsPer2q replicas per CTA, each replica with
// its own shared-memory G and its own named barrier (id 1 + slot, 64 threads)
// instead of block barriers.  The cols/2 pairs of a round are spread over
// groups of lpp lanes (lpp = the largest power of two <= 64 / pairs, at most
// 32, so a group never spans two warps); a group splits the rows of its pair
// and reduces the four dot products with xor shuffles.  Every early return and
// every loop exit depends only on values both warps hold (the replica's
// condition, cols, the shared convergence flags, keep), so both warps reach
// the same barriers.
constexpr int kRepsPer2q = 4;
constexpr int kLanesPerRep = 64;
constexpr int kWarpsPer2q = kRepsPer2q * kLanesPerRep / 32;  // warps per CTA
constexpr uint32_t kWarpCap = 16;

// Largest padded column stride: ld <= 2 cap + 4 when cap is a multiple of 4
// (then 2 cap = 0 mod 8 and lpp >= 4), else <= 2 cap + 7.
__host__ __device__ inline uint32_t warp_ld_max(uint32_t cap) { return 2 * cap + (cap % 4 == 0 ? 4 : 7); }

__host__ __device__ inline uint64_t warp_work_bytes(uint32_t cap) {
  const uint64_t c = 2ull * cap;
  const uint64_t b = c * warp_ld_max(cap) * sizeof(double2) + c * sizeof(double) + c * sizeof(uint32_t);
  return (b + 15) & ~15ull;  // keeps every replica's G 16-byte aligned
}

__device__ __forceinline__ void rep_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

__global__ void __launch_bounds__(kWarpsPer2q * 32) k_mps_2q_warp(MpsView v, uint32_t first, uint32_t max_keep,
                                                                  double thr) {
  const MpsOp& op = v.ops[first + blockIdx.y];
  extern __shared__ double2 smem[];
  __shared__ int s_any[kRepsPer2q][2][2];   // [slot][sweep parity][warp]
  __shared__ uint32_t s_keep[kRepsPer2q];
  __shared__ double s_scale[kRepsPer2q];
  __shared__ double s_n2[kRepsPer2q][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = warp / 2, wr = warp % 2;          // replica slot in the CTA, warp within it
  const uint32_t tl = (uint32_t)(wr * 32 + lane);    // lane within the replica (0..63)
  const int bar = 1 + slot;
  const uint32_t b = blockIdx.x * kRepsPer2q + slot;
  if (b >= v.batch || !cond_ok(v, op, b)) return;    // the same for both warps of the replica
  const unsigned full = 0xffffffffu;
  const uint32_t cap = v.cap;
  uint32_t* dm = v.dims + (uint64_t)b * (v.n + 1);
  const uint32_t q = op.q;
  const uint32_t L = dm[q], M = dm[q + 1], R = dm[q + 2];
  const bool tr = R > L;
  const uint32_t rows = tr ? 2 * R : 2 * L, cols = tr ? 2 * L : 2 * R;
  const uint32_t np = cols / 2;
  uint32_t lpp = 1;  // lanes per pair
  while (lpp < 32 && lpp * 2 * np <= (uint32_t)kLanesPerRep) lpp *= 2;
  // Column stride ld = lpp (mod 8) for lpp < 8: the 8 lanes of a 16-byte access
  // phase (8 / lpp pairs with consecutive columns, lpp rows each) then fall in
  // 8 distinct groups of 4 banks.
  const uint32_t ld = lpp < 8 ? rows + ((lpp + 8 - rows % 8) % 8) : rows;
  const uint32_t tw = 2 * R;
  double2* TH = v.scratch + ((uint64_t)b * v.slots + blockIdx.y) * v.scratch_elems;
  double2* G = reinterpret_cast<double2*>(reinterpret_cast<char*>(smem) + slot * warp_work_bytes(cap));
  double* sig = reinterpret_cast<double*>(G + 2ull * cap * warp_ld_max(cap));
  uint32_t* perm = reinterpret_cast<uint32_t*>(sig + 2 * cap);
  double2* A = site(v, q, b);
  double2* B = site(v, q + 1, b);
  const double2 zero = make_double2(0.0, 0.0);

  double n2loc = 0.0;  // |theta|_F^2, for the negligible-pair test
  for (uint32_t t = tl; t < L * R; t += kLanesPerRep) {
    const uint32_t l = t / R, r = t - (t / R) * R;
    double2 in[4];
    for (int i0 = 0; i0 < 2; ++i0)
      for (int i1 = 0; i1 < 2; ++i1) {
        double2 acc = zero;
        const double2* ar = A + (uint64_t)(l * 2 + i0) * cap;
        for (uint32_t k = 0; k < M; ++k)
          acc = cadd_x(acc, cmul_x(ar[k], B[(uint64_t)(k * 2 + i1) * cap + r]));
        in[i0 * 2 + i1] = acc;
      }
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1) {
        const int o = o0 * 2 + o1;
        double2 acc = zero;
        for (int i = 0; i < 4; ++i) acc = cadd_x(acc, cmul_x(op.u[o * 4 + i], in[i]));
        const uint32_t row = l * 2 + o0, col = o1 * R + r;
        TH[(uint64_t)row * tw + col] = acc;
        n2loc += acc.x * acc.x + acc.y * acc.y;
        if (!tr) G[col * ld + row] = acc;
        else G[row * ld + col] = make_double2(acc.x, -acc.y);
      }
  }
  n2loc = warp_sum(n2loc);
  if (lane == 0) s_n2[slot][wr] = n2loc;
  rep_sync(bar);

  const double tol = (double)rows * DBL_EPSILON;
  const double neg = tol * tol * (s_n2[slot][0] + s_n2[slot][1]);
  const uint32_t pi = tl / lpp, h = tl % lpp;
  const bool active = pi < np;
  for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
    bool rot = false;
    for (uint32_t rd = 0; rd + 1 < cols; ++rd) {
      uint32_t p = 0, qq = 0;
      if (active) {
        if (pi == 0) {
          p = rd;
          qq = cols - 1;
        } else {
          p = (rd + pi) % (cols - 1);
          qq = (rd + (cols - 1) - pi) % (cols - 1);
        }
      }
      double2* gp = G + p * ld;
      double2* gq = G + qq * ld;
      double al = 0.0, be = 0.0, gr = 0.0, gi = 0.0;
      if (active)
        for (uint32_t i = h; i < rows; i += lpp) {
          const double2 x = gp[i], y = gq[i];
          al += x.x * x.x + x.y * x.y;
          be += y.x * y.x + y.y * y.y;
          gr += x.x * y.x + x.y * y.y;
          gi += x.x * y.y - x.y * y.x;
        }
      for (uint32_t o = lpp / 2; o >= 1; o >>= 1) {
        al += __shfl_xor_sync(full, al, o);
        be += __shfl_xor_sync(full, be, o);
        gr += __shfl_xor_sync(full, gr, o);
        gi += __shfl_xor_sync(full, gi, o);
      }
      double c, s, ex, ey;
      if (active && jacobi_rotation(al, be, gr, gi, tol, neg, c, s, ex, ey)) {
        rot = true;
        for (uint32_t i = h; i < rows; i += lpp) {
          const double2 x = gp[i], y = gq[i];
          gp[i] = make_double2(c * x.x - s * (ex * y.x + ey * y.y), c * x.y - s * (ex * y.y - ey * y.x));
          gq[i] = make_double2(s * (ex * x.x - ey * x.y) + c * y.x, s * (ex * x.y + ey * x.x) + c * y.y);
        }
      }
      rep_sync(bar);
    }
    // both warps stop together: each posts its vote, the decision is the OR
    const int vote = __any_sync(full, rot) ? 1 : 0;
    if (lane == 0) s_any[slot][sweep & 1][wr] = vote;
    rep_sync(bar);
    if (!(s_any[slot][sweep & 1][0] | s_any[slot][sweep & 1][1])) break;
  }

  for (uint32_t j = tl; j < cols; j += kLanesPerRep) {
    const double2* g = G + j * ld;
    double sq = 0.0;
    for (uint32_t i = 0; i < rows; ++i) sq += g[i].x * g[i].x + g[i].y * g[i].y;
    sig[j] = sqrt(sq);
  }
  rep_sync(bar);
  for (uint32_t j = tl; j < cols; j += kLanesPerRep) {
    uint32_t rank = 0;
    const double sj = sig[j];
    for (uint32_t i = 0; i < cols; ++i) rank += (sig[i] > sj || (sig[i] == sj && i < j)) ? 1u : 0u;
    perm[rank] = j;
  }
  rep_sync(bar);
  if (tl == 0) {
    uint32_t keep = 0;
    for (uint32_t k = 0; k < cols; ++k) keep += sig[perm[k]] > thr ? 1u : 0u;
    keep = keep > 1u ? keep : 1u;
    if (max_keep) keep = keep < max_keep ? keep : max_keep;
    double kept = 0.0, total = 0.0, disc = 0.0;
    for (uint32_t k = 0; k < keep; ++k) kept += sig[perm[k]] * sig[perm[k]];
    for (uint32_t k = 0; k < cols; ++k) total += sig[perm[k]] * sig[perm[k]];
    for (uint32_t k = keep; k < cols; ++k) disc += sig[perm[k]] * sig[perm[k]];
    kept = fmax(sqrt(kept), 1e-15);
    total = sqrt(total);
    s_scale[slot] = disc > 0.0 ? total / kept : 1.0;
    s_keep[slot] = keep;
    if (keep > cap) {
      atomicMax(&v.flags[2], (int)keep);
      atomicMax(&v.flags[0], MF_CAPACITY);
    } else {
      atomicAdd(v.svd_calls, 1ull);
    }
  }
  rep_sync(bar);
  const uint32_t keep = s_keep[slot];
  const double scale = s_scale[slot];
  if (keep > cap) return;  // the same for both warps

  for (uint32_t t = tl; t < L * 2 * keep; t += kLanesPerRep) {
    const uint32_t row = t / keep, k = t - (t / keep) * keep;
    const uint32_t j = perm[k];
    const double sj = sig[j];
    double2 val = zero;
    if (sj > 0.0 && sj * sj > neg) {  // a kept column at the rounding level of theta is left zero
      if (!tr) {
        const double2 g = G[j * ld + row];
        val = make_double2(g.x / sj, g.y / sj);
      } else {
        const double2* th = TH + (uint64_t)row * tw;
        const double2* w = G + j * ld;
        double re = 0.0, im = 0.0;
        for (uint32_t c2 = 0; c2 < tw; ++c2) {
          const double2 a = th[c2], x = w[c2];
          re += a.x * x.x - a.y * x.y;
          im += a.x * x.y + a.y * x.x;
        }
        const double s2 = sj * sj;
        val = make_double2(re / s2, im / s2);
      }
    }
    A[(uint64_t)row * cap + k] = val;
  }
  for (uint32_t t = tl; t < keep * 2 * R; t += kLanesPerRep) {
    const uint32_t k = t / (2 * R), col = t - (t / (2 * R)) * (2 * R);
    const uint32_t s = col / R, r = col - (col / R) * R;
    const uint32_t j = perm[k];
    const double sj = sig[j];
    double2 val = zero;
    if (sj > 0.0 && sj * sj > neg) {  // a kept column at the rounding level of theta is left zero
      if (tr) {
        const double2 g = G[j * ld + col];
        val = make_double2(scale * g.x, -scale * g.y);
      } else {
        const double2* w = G + j * ld;
        double re = 0.0, im = 0.0;
        for (uint32_t r2 = 0; r2 < rows; ++r2) {
          const double2 x = w[r2], a = TH[(uint64_t)r2 * tw + col];
          re += x.x * a.x + x.y * a.y;
          im += x.x * a.y - x.y * a.x;
        }
        const double f = scale / sj;
        val = make_double2(f * re, f * im);
      }
    }
    B[(uint64_t)(k * 2 + s) * cap + r] = val;
  }
  if (tl == 0) dm[q + 1] = keep;
}

// p1 of qubit op.q by transfer matrices E_{j+1} = sum_s A_j[s]^H E_j A_j[s]
// (s = 1 only at the measured site), then the draw, the projection
// (project_qubit, simulator.rs:276-291), the reset flip and the cbit.
__global__ void __launch_bounds__(kMpsThreads) k_mps_measure(MpsView v, uint32_t first, int use_smem) {
  const MpsOp& op = v.ops[first];
  extern __shared__ double2 smem[];
  __shared__ int s_out;
  __shared__ double s_scale;
  const uint32_t b = blockIdx.x;
  if (!cond_ok(v, op, b)) return;
  const uint32_t* dm = v.dims + (uint64_t)b * (v.n + 1);
  const uint32_t cap = v.cap;
  double2* E = use_smem ? smem : v.scratch + (uint64_t)b * v.slots * v.scratch_elems + theta_elems(v.cap);
  double2* F = E + (uint64_t)cap * cap;
  double2* E2 = F + (uint64_t)cap * cap;
  const double2 zero = make_double2(0.0, 0.0);
  const int tid = threadIdx.x;
  if (tid == 0) E[0] = make_double2(1.0, 0.0);
  __syncthreads();
  for (uint32_t j = 0; j < v.n; ++j) {
    const uint32_t Lj = dm[j], Rj = dm[j + 1];
    const double2* A = site(v, j, b);
    for (uint32_t t = tid; t < Rj * Rj; t += blockDim.x) E2[t] = zero;
    for (int s = 0; s < 2; ++s) {
      if (j == op.q && s == 0) continue;
      __syncthreads();
      // F[l][r'] = sum_l' E[l][l'] A[l'][s][r']
      for (uint32_t t = tid; t < Lj * Rj; t += blockDim.x) {
        const uint32_t l = t / Rj, rp = t - (t / Rj) * Rj;
        double2 acc = zero;
        for (uint32_t lp = 0; lp < Lj; ++lp) {
          const double2 e = E[l * Lj + lp], a = A[(uint64_t)(lp * 2 + s) * cap + rp];
          acc.x += e.x * a.x - e.y * a.y;
          acc.y += e.x * a.y + e.y * a.x;
        }
        F[t] = acc;
      }
      __syncthreads();
      // E2[r][r'] += sum_l conj(A[l][s][r]) F[l][r']
      for (uint32_t t = tid; t < Rj * Rj; t += blockDim.x) {
        const uint32_t r = t / Rj, rp = t - (t / Rj) * Rj;
        double2 acc = E2[t];
        for (uint32_t l = 0; l < Lj; ++l) {
          const double2 a = A[(uint64_t)(l * 2 + s) * cap + r], f = F[l * Rj + rp];
          acc.x += a.x * f.x + a.y * f.y;
          acc.y += a.x * f.y - a.y * f.x;
        }
        E2[t] = acc;
      }
    }
    __syncthreads();
    for (uint32_t t = tid; t < Rj * Rj; t += blockDim.x) E[t] = E2[t];
    __syncthreads();
  }
  if (tid == 0) {
    double p1 = E[0].x;
    p1 = fmin(fmax(p1, 0.0), 1.0);
    const double r = chacha8_draw(v.key + (uint64_t)b * 8, v.ctr[b]);
    v.ctr[b] += 1;
    const int outcome = r < p1 ? 1 : 0;
    const double prob = outcome ? p1 : 1.0 - p1;
    s_out = outcome;
    s_scale = prob > 0.0 ? 1.0 / sqrt(prob) : 0.0;
    if (op.kind == M_MEAS && op.cbit >= 0) v.cbits[(uint64_t)b * v.ncb + op.cbit] = outcome;
  }
  __syncthreads();
  const int outcome = s_out;
  const double2 sc = make_double2(s_scale, 0.0);
  double2* A = site(v, op.q, b);
  const uint32_t L = dm[op.q], R = dm[op.q + 1];
  for (uint32_t t = tid; t < L * 2 * R; t += blockDim.x) {
    const uint32_t row = t / R, r = t - (t / R) * R;   // row = l*2 + s
    double2* p = A + (uint64_t)row * cap + r;
    *p = ((int)(row & 1u) == outcome) ? cmul_x(*p, sc) : zero;
  }
  if (op.kind == M_RESET && outcome == 1) {
    __syncthreads();
    const double2 xm[4] = {zero, make_double2(1.0, 0.0), make_double2(1.0, 0.0), zero};
    site_1q(A, L, R, cap, xm);
  }
}

// Batched form of k_mps_measure for capacity <= 16: two warps per replica
// (joined by the replica's named barrier, as in k_mps_2q_warp), kRepsPer2q
// replicas per CTA; the three transfer matrices of a replica (3 x cap^2) live in
// its slice of shared memory.
__host__ __device__ inline uint64_t warp_measure_bytes(uint32_t cap) {
  return 3ull * cap * cap * sizeof(double2);
}

__global__ void __launch_bounds__(kWarpsPer2q * 32) k_mps_measure_warp(MpsView v, uint32_t first) {
  const MpsOp& op = v.ops[first];
  extern __shared__ double2 smem[];
  __shared__ int s_out[kRepsPer2q];
  __shared__ double s_sc[kRepsPer2q];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = warp / 2, wr = warp % 2;
  const uint32_t tl = (uint32_t)(wr * 32 + lane);
  const int bar = 1 + slot;
  const uint32_t b = blockIdx.x * kRepsPer2q + slot;
  if (b >= v.batch || !cond_ok(v, op, b)) return;  // the same for both warps of the replica
  const uint32_t* dm = v.dims + (uint64_t)b * (v.n + 1);
  const uint32_t cap = v.cap;
  double2* E = smem + (uint64_t)slot * 3 * cap * cap;
  double2* F = E + (uint64_t)cap * cap;
  double2* E2 = F + (uint64_t)cap * cap;
  const double2 zero = make_double2(0.0, 0.0);
  if (tl == 0) E[0] = make_double2(1.0, 0.0);
  rep_sync(bar);
  for (uint32_t j = 0; j < v.n; ++j) {
    const uint32_t Lj = dm[j], Rj = dm[j + 1];
    const double2* A = site(v, j, b);
    for (uint32_t t = tl; t < Rj * Rj; t += kLanesPerRep) E2[t] = zero;
    for (int s = 0; s < 2; ++s) {
      if (j == op.q && s == 0) continue;
      rep_sync(bar);
      for (uint32_t t = tl; t < Lj * Rj; t += kLanesPerRep) {
        const uint32_t l = t / Rj, rp = t - (t / Rj) * Rj;
        double2 acc = zero;
        for (uint32_t lp = 0; lp < Lj; ++lp) {
          const double2 e = E[l * Lj + lp], a = A[(uint64_t)(lp * 2 + s) * cap + rp];
          acc.x += e.x * a.x - e.y * a.y;
          acc.y += e.x * a.y + e.y * a.x;
        }
        F[t] = acc;
      }
      rep_sync(bar);
      for (uint32_t t = tl; t < Rj * Rj; t += kLanesPerRep) {
        const uint32_t r = t / Rj, rp = t - (t / Rj) * Rj;
        double2 acc = E2[t];
        for (uint32_t l = 0; l < Lj; ++l) {
          const double2 a = A[(uint64_t)(l * 2 + s) * cap + r], f = F[l * Rj + rp];
          acc.x += a.x * f.x + a.y * f.y;
          acc.y += a.x * f.y - a.y * f.x;
        }
        E2[t] = acc;
      }
    }
    rep_sync(bar);
    for (uint32_t t = tl; t < Rj * Rj; t += kLanesPerRep) E[t] = E2[t];
    rep_sync(bar);
  }
  if (tl == 0) {
    const double p1 = fmin(fmax(E[0].x, 0.0), 1.0);
    const double r = chacha8_draw(v.key + (uint64_t)b * 8, v.ctr[b]);
    v.ctr[b] += 1;
    const int outcome = r < p1 ? 1 : 0;
    const double prob = outcome ? p1 : 1.0 - p1;
    s_out[slot] = outcome;
    s_sc[slot] = prob > 0.0 ? 1.0 / sqrt(prob) : 0.0;
    if (op.kind == M_MEAS && op.cbit >= 0) v.cbits[(uint64_t)b * v.ncb + op.cbit] = outcome;
  }
  rep_sync(bar);
  const int outcome = s_out[slot];
  const double2 sc = make_double2(s_sc[slot], 0.0);
  double2* A = site(v, op.q, b);
  const uint32_t L = dm[op.q], R = dm[op.q + 1];
  for (uint32_t t = tl; t < L * 2 * R; t += kLanesPerRep) {
    const uint32_t row = t / R, r = t - (t / R) * R;
    double2* p = A + (uint64_t)row * cap + r;
    *p = ((int)(row & 1u) == outcome) ? cmul_x(*p, sc) : zero;
  }
  if (op.kind == M_RESET && outcome == 1) {
    rep_sync(bar);
    const double2 x1 = make_double2(1.0, 0.0);
    for (uint32_t t = tl; t < L * R; t += kLanesPerRep) {
      const uint32_t l = t / R, r = t - (t / R) * R;
      double2* p0 = A + (uint64_t)(l * 2) * cap + r;
      double2* p1 = p0 + cap;
      const double2 a0 = *p0, a1 = *p1;
      *p0 = cadd_x(cadd_x(zero, cmul_x(zero, a0)), cmul_x(x1, a1));
      *p1 = cadd_x(cadd_x(zero, cmul_x(x1, a0)), cmul_x(zero, a1));
    }
  }
}

__global__ void k_mps_fail(MpsView v, uint32_t first) {
  const MpsOp& op = v.ops[first];
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.batch || !cond_ok(v, op, b)) return;
  atomicMax(&v.flags[0], MF_UNSUPPORTED);
  atomicMin(&v.flags[1], op.inst);
}

// One site of to_statevector (simulator.rs:238-257): from W (2^k x Lk, row i
// = basis bits of qubits 0..k-1) to W' (2^(k+1) x Rk): W'[i + s 2^k][r] =
// sum_l W[i][l] A[l][s][r], accumulated from zero in ascending l.
__global__ void __launch_bounds__(256) k_mps_expand(const double2* __restrict__ w,
                                                    double2* __restrict__ wn,
                                                    const double2* __restrict__ a, uint32_t k,
                                                    uint32_t Lk, uint32_t Rk, uint32_t cap) {
  const uint64_t total = (2ull << k) * Rk;
  const uint64_t half = 1ull << k;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i2 = t / Rk;
    const uint32_t r = (uint32_t)(t - i2 * Rk);
    const uint64_t i = i2 & (half - 1);
    const uint32_t s = (uint32_t)(i2 >> k);
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t l = 0; l < Lk; ++l)
      acc = cadd_x(acc, cmul_x(w[i * Lk + l], a[(uint64_t)(l * 2 + s) * cap + r]));
    wn[t] = acc;
  }
}

// ---- host side -------------------------------------------------------------------

bool is_two_qubit_kind(int kind) {
  switch (kind) {
    case DQ_CX: case DQ_CZ: case DQ_CY: case DQ_CH: case DQ_SWAP: case DQ_CSX: case DQ_CRX:
    case DQ_CRY: case DQ_CRZ: case DQ_CU1: case DQ_CP: case DQ_CU3: case DQ_CU: case DQ_RXX:
    case DQ_RZZ: case DQ_G_PHI_PLUS: case DQ_G_PSI_MINUS: case DQ_G_PSI_PLUS: case DQ_G_CZ:
    case DQ_G_CX:
      return true;
    default:
      return false;
  }
}

void set_u(MpsOp& op, const hc* m, int count) {
  for (int i = 0; i < count; ++i) op.u[i] = make_double2(m[i].re, m[i].im);
}

// reverse_2q_order (simulator.rs:561-579): the gate with its two qubits exchanged.
void reverse_2q(const hc in[16], hc out[16]) {
  for (int a0 = 0; a0 < 2; ++a0)
    for (int b0 = 0; b0 < 2; ++b0)
      for (int a1 = 0; a1 < 2; ++a1)
        for (int b1 = 0; b1 < 2; ++b1)
          out[(a0 * 2 + b0) * 4 + (a1 * 2 + b1)] = in[(b0 * 2 + a0) * 4 + (b1 * 2 + a1)];
}

}  // namespace
}  // namespace dq

using namespace dq;

struct dq_mps_s {
  int device = 0;
  uint32_t n = 0;
  uint32_t batch = 0;
  uint32_t cap = 0;
  uint32_t max_bond = 0;    // 0 = unbounded
  double thr = 1e-12;
  uint32_t ncb = 0;
  cudaStream_t stream = nullptr;
  double2* t = nullptr;
  uint32_t* dims = nullptr;
  uint32_t* key = nullptr;
  unsigned long long* ctr = nullptr;
  int32_t* cbits = nullptr;
  dq_cond* conds = nullptr;
  uint64_t conds_cap = 0;
  double2* scratch = nullptr;
  int* flags = nullptr;
  unsigned long long* svd_calls = nullptr;
  bool broken = false;       // a failed reserve lost the state: every later call fails
  size_t buf_bytes[8] = {};  // sizes of t, dims, key, ctr, cbits, flags, svd_calls, scratch
  bool smem = true;
  uint64_t scratch_elems = 0;
  size_t work_bytes = 0;
  uint32_t slots = 1;        // two-qubit steps one launch may run per replica
  void* ops = nullptr;       // device copy of the program's operations
  size_t ops_cap = 0;
};

namespace {

uint32_t bond_bound(uint32_t n, uint32_t max_bond) {
  const uint32_t half = n / 2;
  const uint64_t b = half >= 31 ? (1ull << 31) : (1ull << half);
  uint64_t r = b < 1 ? 1 : b;
  if (max_bond && max_bond < r) r = max_bond;
  return (uint32_t)r;
}

// The batch buffers come from the engine's size-keyed device buffer cache:
// repeated shot runs and simulations of one shape pay no cudaMalloc / cudaFree
// (a shot run creates and destroys its handle every call).
void** mps_buf(dq_mps_s* h, int i) {
  void** p[8] = {(void**)&h->t, (void**)&h->dims, (void**)&h->key, (void**)&h->ctr,
                 (void**)&h->cbits, (void**)&h->flags, (void**)&h->svd_calls, (void**)&h->scratch};
  return p[i];
}

int mps_take(dq_mps_s* h, int i, size_t bytes) {
  bytes = std::max<size_t>(bytes, 16);
  void** p = mps_buf(h, i);
  const int rc = cache_alloc(h->device, bytes, p);
  if (rc != DQ_OK) {
    *p = nullptr;
    return rc;
  }
  h->buf_bytes[i] = bytes;
  return DQ_OK;
}

void free_buffers(dq_mps_s* h) {
  // a cached buffer may be handed out at once: nothing may still use it
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int i = 0; i < 8; ++i) {
    void** p = mps_buf(h, i);
    if (*p) cache_free(h->device, h->buf_bytes[i], *p);
    *p = nullptr;
    h->buf_bytes[i] = 0;
  }
  cudaFree(h->conds);
  cudaFree(h->ops);
  h->ops = nullptr;
  h->ops_cap = 0;
  h->t = nullptr; h->dims = nullptr; h->key = nullptr; h->ctr = nullptr; h->cbits = nullptr;
  h->conds = nullptr; h->scratch = nullptr; h->flags = nullptr; h->svd_calls = nullptr;
  h->conds_cap = 0;
  h->ncb = 0;
}

constexpr size_t kMaxSmem = 220 * 1024;
// Largest bond capacity: one CTA's Jacobi SVD of a 2048 x 2048 theta takes
// on the order of a second.
constexpr uint32_t kMaxCapacity = 1024;

// Steps on disjoint bonds are independent: with few replicas, one launch runs
// up to this many of them per replica (each with its own scratch slot).
uint32_t slots_for(uint32_t n, uint32_t batch) {
  if (batch > 2 * 148) return 1;
  return std::max<uint32_t>(1, std::min<uint32_t>(n / 2, 32));
}

int alloc_buffers(dq_mps_s* h, uint32_t batch, uint32_t cap, uint32_t ncb) {
  free_buffers(h);
  h->batch = batch;
  h->slots = slots_for(h->n, batch);
  h->cap = cap;
  h->ncb = ncb ? ncb : 1;
  const uint64_t site = 2ull * cap * cap;
  const size_t work_bytes = svd_work_elems(cap) * sizeof(double2);
  h->smem = work_bytes <= kMaxSmem;
  h->work_bytes = work_bytes;
  h->scratch_elems = theta_elems(cap) + (h->smem ? 0 : svd_work_elems(cap));
  DQ_TRY(mps_take(h, 0, sizeof(double2) * site * h->n * batch));
  DQ_TRY(mps_take(h, 1, sizeof(uint32_t) * (h->n + 1) * batch));
  DQ_TRY(mps_take(h, 2, sizeof(uint32_t) * 8 * batch));
  DQ_TRY(mps_take(h, 3, sizeof(unsigned long long) * batch));
  DQ_TRY(mps_take(h, 4, sizeof(int32_t) * h->ncb * batch));
  DQ_TRY(mps_take(h, 5, sizeof(int) * 4));
  DQ_TRY(mps_take(h, 6, sizeof(unsigned long long)));
  DQ_TRY(mps_take(h, 7, sizeof(double2) * h->scratch_elems * h->slots * batch));
  if (cap <= kWarpCap)
    DQ_CUDA_TRY(cudaFuncSetAttribute(k_mps_measure_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(kRepsPer2q * warp_measure_bytes(cap))));
  if (cap <= kWarpCap)
    DQ_CUDA_TRY(cudaFuncSetAttribute(k_mps_2q_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(kRepsPer2q * warp_work_bytes(cap))));
  if (h->smem) {
    DQ_CUDA_TRY(cudaFuncSetAttribute(k_mps_2q, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)work_bytes));
    DQ_CUDA_TRY(cudaFuncSetAttribute(k_mps_measure, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)work_bytes));
  }
  return DQ_OK;
}

MpsView view_of(const dq_mps_s* h) {
  MpsView v;
  v.t = h->t;
  v.dims = h->dims;
  v.key = h->key;
  v.ctr = h->ctr;
  v.cbits = h->cbits;
  v.conds = h->conds;
  v.scratch = h->scratch;
  v.flags = h->flags;
  v.svd_calls = h->svd_calls;
  v.ops = static_cast<const MpsOp*>(h->ops);
  v.slots = h->slots;
  v.site_elems = 2ull * h->cap * h->cap;
  v.scratch_elems = h->scratch_elems;
  v.n = h->n;
  v.batch = h->batch;
  v.cap = h->cap;
  v.ncb = h->ncb;
  return v;
}

// Lowers the program into batch operations (run_instruction, simulator.rs:457-559).
// Returns DQ_ERR_UNSUPPORTED with *failed set for an unconditional operation
// the MPS simulator rejects; conditional ones become M_FAIL operations.
int lower(uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_cond* conds, uint64_t nconds,
          uint64_t ncbits, std::vector<MpsOp>& ops, int64_t* failed) {
  ops.clear();
  for (uint64_t i = 0; i < ninst; ++i) {
    const dq_inst& in = prog[i];
    MpsOp op;
    memset(&op, 0, sizeof(op));
    op.cond_first = in.cond_first;
    op.cond_count = in.cond_count;
    op.inst = (int32_t)i;
    op.cbit = -1;
    const bool two = is_two_qubit_kind(in.kind);
    if (!(two && in.nq == 2 && in.q[0] == in.q[1]))
      DQ_TRY(validate_inst(in, n, nconds, ncbits, conds, i));
    else if (in.q[0] < 0 || (uint32_t)in.q[0] >= n)
      return fail(DQ_ERR_INVALID_ARG, "instruction " + std::to_string(i) + ": qubit out of range");
    switch (in.kind) {
      case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP: case DQ_G_OPAQUE:
        continue;
      case DQ_MEASURE: case DQ_RESET:
        op.kind = in.kind == DQ_MEASURE ? M_MEAS : M_RESET;
        op.q = (uint32_t)in.q[0];
        op.cbit = in.kind == DQ_MEASURE ? (int32_t)in.cbit : -1;
        ops.push_back(op);
        continue;
      default: break;
    }
    hc m[4];
    if (matrix_1q(in.kind, in.p, m)) {
      op.kind = M_1Q;
      op.q = (uint32_t)in.q[0];
      set_u(op, m, 4);
      ops.push_back(op);
      continue;
    }
    if (two) {
      const uint32_t a = (uint32_t)in.q[0], bq = (uint32_t)in.q[1];
      if (a == bq) continue;  // apply_2q returns early for a == b
      static thread_local Gate g;
      if (!matrix_nq(in, g) || g.k != 2) return fail(DQ_ERR_INTERNAL, "two-qubit kind without a 4x4 matrix");
      hc swapm[16], gm[16];
      {
        dq_inst sw;
        memset(&sw, 0, sizeof(sw));
        sw.kind = DQ_SWAP;
        sw.nq = 2;
        static thread_local Gate gs;
        matrix_nq(sw, gs);
        for (int k = 0; k < 16; ++k) swapm[k] = gs.m[k];
      }
      const uint32_t lo = a < bq ? a : bq, hi = a < bq ? bq : a;
      if (a < bq) for (int k = 0; k < 16; ++k) gm[k] = g.m[k];
      else reverse_2q(g.m, gm);
      MpsOp s = op;
      s.kind = M_2Q;
      set_u(s, swapm, 16);
      for (uint32_t pos = hi - 1; pos > lo; --pos) {
        s.q = pos;
        ops.push_back(s);
      }
      MpsOp gop = op;
      gop.kind = M_2Q;
      gop.q = lo;
      set_u(gop, gm, 16);
      ops.push_back(gop);
      for (uint32_t pos = lo + 1; pos < hi; ++pos) {
        s.q = pos;
        ops.push_back(s);
      }
      continue;
    }
    // generic names the MPS dispatcher rejects, and gates on three or more qubits
    if (in.cond_count == 0) {
      *failed = (int64_t)i;
      return fail(DQ_ERR_UNSUPPORTED, "instruction " + std::to_string(i) + " is not supported by the MPS simulator");
    }
    op.kind = M_FAIL;
    ops.push_back(op);
  }
  return DQ_OK;
}

// Groups consecutive operations into launches: a run of one-qubit gates, or
// of two-qubit steps (at most `slots`), whose sites are pairwise disjoint
// commutes exactly, so one launch (blockIdx.y = the operation) runs them all;
// measurements, resets and failures are launches of their own.
int launch_ops(dq_mps_s* h, const std::vector<MpsOp>& ops) {
  if (ops.empty()) return DQ_OK;
  if (ops.size() > h->ops_cap) {
    cudaFree(h->ops);
    h->ops = nullptr;
    h->ops_cap = 0;
    DQ_CUDA_TRY(cudaMalloc(&h->ops, sizeof(MpsOp) * ops.size()));
    h->ops_cap = ops.size();
  }
  DQ_CUDA_TRY(cudaMemcpyAsync(h->ops, ops.data(), sizeof(MpsOp) * ops.size(), cudaMemcpyHostToDevice,
                              h->stream));
  const MpsView v = view_of(h);
  const size_t shm = h->smem ? h->work_bytes : 0;
  const int use = h->smem ? 1 : 0;
  // one SVD per CTA: wide CTAs when few replicas share the GPU (latency), 256
  // threads and several CTAs per SM otherwise (throughput)
  const int t2q = h->batch <= 2 * 148 ? 1024 : 256;
  // many replicas of small bonds: one warp per replica
  const bool warp2q = h->batch > 2 * 148 && h->cap <= kWarpCap;
  std::vector<uint8_t> used(h->n, 0);
  for (size_t i = 0; i < ops.size();) {
    const int kind = ops[i].kind;
    size_t j = i;
    if (kind == M_1Q || kind == M_2Q) {
      std::fill(used.begin(), used.end(), 0);
      const size_t limit = kind == M_2Q ? h->slots : 65535;
      while (j < ops.size() && ops[j].kind == kind && j - i < limit) {
        const uint32_t q = ops[j].q, q2 = kind == M_2Q ? q + 1 : q;
        if (used[q] || used[q2]) break;
        used[q] = used[q2] = 1;
        ++j;
      }
    } else {
      j = i + 1;
    }
    const uint32_t first = (uint32_t)i, count = (uint32_t)(j - i);
    switch (kind) {
      case M_1Q: k_mps_1q<<<dim3(h->batch, count), kMpsThreads, 0, h->stream>>>(v, first); break;
      case M_2Q:
        if (warp2q)
          k_mps_2q_warp<<<dim3((h->batch + kRepsPer2q - 1) / kRepsPer2q, count), kWarpsPer2q * 32,
                          kRepsPer2q * warp_work_bytes(h->cap), h->stream>>>(v, first, h->max_bond, h->thr);
        else
          k_mps_2q<<<dim3(h->batch, count), t2q, shm, h->stream>>>(v, first, h->max_bond, h->thr, use);
        break;
      case M_MEAS: case M_RESET:
        if (warp2q)
          k_mps_measure_warp<<<(h->batch + kRepsPer2q - 1) / kRepsPer2q, kWarpsPer2q * 32,
                               kRepsPer2q * warp_measure_bytes(h->cap), h->stream>>>(v, first);
        else
          k_mps_measure<<<h->batch, kMpsThreads, shm, h->stream>>>(v, first, use);
        break;
      case M_FAIL: k_mps_fail<<<(h->batch + 127) / 128, 128, 0, h->stream>>>(v, first); break;
      default: return fail(DQ_ERR_INTERNAL, "bad MPS operation");
    }
    i = j;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(DQ_ERR_CUDA, std::string("MPS launch: ") + cudaGetErrorString(e));
  return DQ_OK;
}

// Runs `ops` on a batch whose replica b is seeded with seeds[b]; grows the
// capacity and re-runs while a truncation overflows it.
uint64_t replica_bytes(uint32_t n, uint32_t cap, uint32_t slots) {
  const uint64_t work = svd_work_elems(cap) * sizeof(double2);
  return (uint64_t)n * 2ull * cap * cap * sizeof(double2) +
         slots * (theta_elems(cap) * sizeof(double2) + (work <= kMaxSmem ? 0 : work));
}

// Runs `ops` on a batch whose replica b is seeded with seeds[b]; grows the
// capacity and re-runs while a truncation overflows it.  With batch > 1 and a
// grown capacity whose buffers would exceed `budget` bytes, it returns with
// *shrink set (and the new capacity recorded) so that the caller re-splits.
int run_batch(dq_mps_s* h, const std::vector<MpsOp>& ops, const dq_cond* conds, uint64_t nconds,
              const uint64_t* seeds, uint32_t batch, uint32_t ncb, int* status, int* failed_inst,
              double* kernel_ms, uint64_t budget = 0, bool* shrink = nullptr) {
  const uint32_t bound = bond_bound(h->n, h->max_bond);
  if (shrink) *shrink = false;
  for (;;) {
    if (h->batch != batch || h->ncb != (ncb ? ncb : 1) || !h->t) DQ_TRY(alloc_buffers(h, batch, h->cap, ncb));
    if (nconds > h->conds_cap) {
      cudaFree(h->conds);
      h->conds = nullptr;
      DQ_CUDA_TRY(cudaMalloc((void**)&h->conds, sizeof(dq_cond) * nconds));
      h->conds_cap = nconds;
    }
    if (nconds)
      DQ_CUDA_TRY(cudaMemcpyAsync(h->conds, conds, sizeof(dq_cond) * nconds, cudaMemcpyHostToDevice, h->stream));
    std::vector<uint32_t> keys((size_t)batch * 8);
    for (uint32_t b = 0; b < batch; ++b) seed_key_from_u64(seeds[b], &keys[(size_t)b * 8]);
    DQ_CUDA_TRY(cudaMemcpyAsync(h->key, keys.data(), sizeof(uint32_t) * keys.size(), cudaMemcpyHostToDevice,
                                h->stream));
    const int init_flags[4] = {MF_OK, 0x7fffffff, 0, 0};
    DQ_CUDA_TRY(cudaMemcpyAsync(h->flags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, h->stream));
    DQ_CUDA_TRY(cudaMemsetAsync(h->svd_calls, 0, sizeof(unsigned long long), h->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, h->stream);
    k_mps_reset<<<batch, kMpsThreads, 0, h->stream>>>(view_of(h));
    int rc = launch_ops(h, ops);
    cudaEventRecord(e1, h->stream);
    int fl[4] = {0, 0, 0, 0};
    if (rc == DQ_OK) {
      const cudaError_t e = cudaMemcpyAsync(fl, h->flags, sizeof(fl), cudaMemcpyDeviceToHost, h->stream);
      const cudaError_t s = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess || s != cudaSuccess)
        rc = fail(DQ_ERR_CUDA, std::string("MPS run: ") + cudaGetErrorString(e != cudaSuccess ? e : s));
    }
    float ms = 0.f;
    if (rc == DQ_OK) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != DQ_OK) return rc;
    if (fl[0] == MF_CAPACITY) {
      uint32_t need = (uint32_t)fl[2];
      uint32_t cap = h->cap;
      while (cap < need) cap *= 2;
      if (cap > bound) cap = bound;
      if (cap <= h->cap) return fail(DQ_ERR_INTERNAL, "MPS bond dimension above its bound");
      if (cap > kMaxCapacity)
        return fail(DQ_ERR_INVALID_ARG, "bond dimension " + std::to_string(need) +
                                            " exceeds the device MPS limit of " +
                                            std::to_string(kMaxCapacity) + "; set max_bond_dimension");
      if (shrink && batch > 1 && budget && replica_bytes(h->n, cap, slots_for(h->n, batch)) * batch > budget) {
        free_buffers(h);
        h->cap = cap;
        *shrink = true;
        return DQ_OK;
      }
      DQ_TRY(alloc_buffers(h, batch, cap, ncb));
      continue;
    }
    *status = fl[0];
    *failed_inst = fl[1];
    if (kernel_ms) *kernel_ms = ms;
    return DQ_OK;
  }
}

int check_mps(dq_mps_t h) {
  if (!h || !h->stream) return fail(DQ_ERR_INVALID_ARG, "null or destroyed MPS handle");
  if (h->broken) return fail(DQ_ERR_INVALID_ARG, "MPS handle lost its state in a failed reserve");
  return DQ_OK;
}

int new_handle(uint32_t n, int device, uint32_t max_bond, double thr, dq_mps_s** out) {
  if (n == 0 || n > 64) return fail(DQ_ERR_INVALID_ARG, "MPS qubit count must be in [1, 64]");
  // any threshold is accepted, as MpsSimulator::new does: a negative one keeps
  // every singular value, NaN or +inf keeps one (s > thr is false)
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(DQ_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= count) return fail(DQ_ERR_INVALID_ARG, "bad device ordinal");
  DeviceGuard g(device);
  dq_mps_s* h = new dq_mps_s();
  h->device = device;
  h->n = n;
  h->max_bond = max_bond;
  h->thr = thr;
  h->cap = std::min<uint32_t>(bond_bound(n, max_bond), 16u);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return fail(DQ_ERR_CUDA, "cudaStreamCreate failed");
  }
  *out = h;
  return DQ_OK;
}

void destroy_handle(dq_mps_s* h) {
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  free_buffers(h);
  cudaStreamDestroy(h->stream);
  h->stream = nullptr;
  delete h;
}

int map_status(int status, int failed, int64_t* out_failed) {
  if (status == MF_UNSUPPORTED) {
    if (out_failed) *out_failed = failed;
    return fail(DQ_ERR_UNSUPPORTED, "instruction " + std::to_string(failed) +
                                        " is not supported by the MPS simulator");
  }
  if (status != MF_OK) return fail(DQ_ERR_INTERNAL, "MPS run flagged status " + std::to_string(status));
  return DQ_OK;
}

}  // namespace

extern "C" {

int dq_mps_create(uint32_t n, int device, uint32_t max_bond, double truncation_threshold, dq_mps_t* out) {
  clear_error();
  if (!out) return fail(DQ_ERR_INVALID_ARG, "null output handle");
  *out = nullptr;
  dq_mps_s* h = nullptr;
  DQ_TRY(new_handle(n, device, max_bond, truncation_threshold, &h));
  DeviceGuard g(device);
  int rc = alloc_buffers(h, 1, h->cap, 1);
  if (rc == DQ_OK) {
    const uint64_t seed = 0;
    std::vector<MpsOp> none;
    int st = 0, fi = 0;
    rc = run_batch(h, none, nullptr, 0, &seed, 1, 1, &st, &fi, nullptr);
  }
  if (rc != DQ_OK) {
    destroy_handle(h);
    return rc;
  }
  *out = h;
  return DQ_OK;
}

int dq_mps_destroy(dq_mps_t h) {
  clear_error();
  if (!h) return DQ_OK;
  destroy_handle(h);
  return DQ_OK;
}

int dq_mps_run(dq_mps_t h, const dq_inst* prog, uint64_t ninst, const dq_cond* conds, uint64_t nconds,
               uint64_t seed, int32_t* cbits, uint64_t ncbits, dq_mps_stats* stats) {
  clear_error();
  DQ_TRY(check_mps(h));
  if ((ninst && !prog) || (nconds && !conds) || (ncbits && !cbits))
    return fail(DQ_ERR_INVALID_ARG, "null program, condition or cbit buffer");
  if (ncbits > (1u << 26)) return fail(DQ_ERR_INVALID_ARG, "classical register array too large");
  if (stats) memset(stats, 0, sizeof(*stats));
  if (stats) stats->failed_inst = -1;
  DeviceGuard g(h->device);
  std::vector<MpsOp> ops;
  int64_t failed = -1;
  int rc = lower(h->n, prog, ninst, conds, nconds, ncbits, ops, &failed);
  if (rc != DQ_OK) {
    if (stats) stats->failed_inst = failed;
    return rc;
  }
  int st = 0, fi = 0;
  double ms = 0.0;
  DQ_TRY(run_batch(h, ops, conds, nconds, &seed, 1, (uint32_t)ncbits, &st, &fi, &ms));
  int64_t f64 = -1;
  rc = map_status(st, fi, &f64);
  if (stats) {
    stats->failed_inst = f64;
    stats->kernel_ms = ms;
    stats->capacity = h->cap;
    stats->replicas = 1;
    unsigned long long calls = 0;
    cudaMemcpy(&calls, h->svd_calls, sizeof(calls), cudaMemcpyDeviceToHost);
    stats->svd_calls = calls;
  }
  if (rc != DQ_OK) return rc;
  if (ncbits) DQ_CUDA_TRY(cudaMemcpy(cbits, h->cbits, sizeof(int32_t) * ncbits, cudaMemcpyDeviceToHost));
  return DQ_OK;
}

int dq_mps_apply_2q(dq_mps_t h, uint32_t a, uint32_t b, const double* u) {
  clear_error();
  DQ_TRY(check_mps(h));
  if (!u || a >= h->n || b >= h->n) return fail(DQ_ERR_INVALID_ARG, "bad qubit or null matrix");
  if (a == b) return DQ_OK;
  DeviceGuard g(h->device);
  hc m[16], swapm[16], gm[16];
  for (int k = 0; k < 16; ++k) m[k] = hc{u[2 * k], u[2 * k + 1]};
  {
    dq_inst sw;
    memset(&sw, 0, sizeof(sw));
    sw.kind = DQ_SWAP;
    sw.nq = 2;
    static thread_local Gate gs;
    matrix_nq(sw, gs);
    for (int k = 0; k < 16; ++k) swapm[k] = gs.m[k];
  }
  if (a < b) for (int k = 0; k < 16; ++k) gm[k] = m[k];
  else reverse_2q(m, gm);
  const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  std::vector<MpsOp> ops;
  MpsOp op;
  memset(&op, 0, sizeof(op));
  op.kind = M_2Q;
  op.cbit = -1;
  op.inst = -1;
  set_u(op, swapm, 16);
  for (uint32_t pos = hi - 1; pos > lo; --pos) { op.q = pos; ops.push_back(op); }
  MpsOp gop = op;
  gop.q = lo;
  set_u(gop, gm, 16);
  ops.push_back(gop);
  for (uint32_t pos = lo + 1; pos < hi; ++pos) { op.q = pos; ops.push_back(op); }
  // Below the bond bound a step may overflow the capacity: run the steps one
  // at a time, and on an overflow (the step wrote nothing) widen and redo it.
  const uint32_t bound = bond_bound(h->n, h->max_bond);
  const int init_flags[4] = {MF_OK, 0x7fffffff, 0, 0};
  if (h->cap >= bound) {
    DQ_CUDA_TRY(cudaMemcpyAsync(h->flags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, h->stream));
    DQ_TRY(launch_ops(h, ops));
    int fl[4];
    DQ_CUDA_TRY(cudaMemcpyAsync(fl, h->flags, sizeof(fl), cudaMemcpyDeviceToHost, h->stream));
    DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return map_status(fl[0], fl[1], nullptr);
  }
  for (size_t i = 0; i < ops.size();) {
    DQ_CUDA_TRY(cudaMemcpyAsync(h->flags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, h->stream));
    DQ_TRY(launch_ops(h, std::vector<MpsOp>(1, ops[i])));
    int fl[4];
    DQ_CUDA_TRY(cudaMemcpyAsync(fl, h->flags, sizeof(fl), cudaMemcpyDeviceToHost, h->stream));
    DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (fl[0] == MF_CAPACITY) {
      uint32_t cap = h->cap;
      while (cap < (uint32_t)fl[2]) cap *= 2;
      DQ_TRY(dq_mps_reserve(h, cap < bound ? cap : bound));
      continue;
    }
    DQ_TRY(map_status(fl[0], fl[1], nullptr));
    ++i;
  }
  return DQ_OK;
}

int dq_mps_reserve(dq_mps_t h, uint32_t capacity) {
  clear_error();
  DQ_TRY(check_mps(h));
  const uint32_t bound = bond_bound(h->n, h->max_bond);
  if (capacity == 0 || capacity > bound || capacity > kMaxCapacity)
    return fail(DQ_ERR_INVALID_ARG, "capacity must be in [1, " +
                                        std::to_string(std::min(bound, kMaxCapacity)) + "]");
  if (capacity <= h->cap) return DQ_OK;
  if (h->batch != 1) return fail(DQ_ERR_INVALID_ARG, "dq_mps_reserve takes a single-state handle");
  DeviceGuard g(h->device);
  // keep the current state: copy every site into the larger layout
  const uint32_t old = h->cap, n = h->n;
  std::vector<double2> host((size_t)n * 2 * old * old);
  DQ_CUDA_TRY(cudaMemcpyAsync(host.data(), h->t, sizeof(double2) * host.size(), cudaMemcpyDeviceToHost, h->stream));
  std::vector<uint32_t> dims(n + 1);
  DQ_CUDA_TRY(cudaMemcpyAsync(dims.data(), h->dims, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, h->stream));
  std::vector<unsigned long long> ctr(1);
  DQ_CUDA_TRY(cudaMemcpyAsync(ctr.data(), h->ctr, sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
  std::vector<uint32_t> key(8);
  DQ_CUDA_TRY(cudaMemcpyAsync(key.data(), h->key, sizeof(uint32_t) * 8, cudaMemcpyDeviceToHost, h->stream));
  DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const uint32_t ncb = h->ncb;
  uint32_t cap = capacity;
  int rc = alloc_buffers(h, 1, capacity, ncb);
  if (rc != DQ_OK) {
    // The wider buffers could not be had (alloc_buffers freed the old ones
    // first): put the state back at its old capacity from the host copy, so
    // the handle stays usable and the caller sees the allocation error.
    const std::string why = dq_last_error();
    if (alloc_buffers(h, 1, old, ncb) != DQ_OK) {
      free_buffers(h);
      h->broken = true;
      return fail(rc, why + " (the MPS state could not be restored: the handle is unusable)");
    }
    cap = old;
  }
  std::vector<double2> wide((size_t)n * 2 * cap * cap, make_double2(0.0, 0.0));
  for (uint32_t k = 0; k < n; ++k)
    for (uint32_t row = 0; row < 2 * old; ++row)
      for (uint32_t r = 0; r < old; ++r)
        wide[(size_t)k * 2 * cap * cap + (size_t)row * cap + r] =
            host[(size_t)k * 2 * old * old + (size_t)row * old + r];
  DQ_CUDA_TRY(cudaMemcpyAsync(h->t, wide.data(), sizeof(double2) * wide.size(), cudaMemcpyHostToDevice, h->stream));
  DQ_CUDA_TRY(cudaMemcpyAsync(h->dims, dims.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, h->stream));
  DQ_CUDA_TRY(cudaMemcpyAsync(h->ctr, ctr.data(), sizeof(unsigned long long), cudaMemcpyHostToDevice, h->stream));
  DQ_CUDA_TRY(cudaMemcpyAsync(h->key, key.data(), sizeof(uint32_t) * 8, cudaMemcpyHostToDevice, h->stream));
  DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (rc != DQ_OK) {
    const std::string why = dq_last_error();
    return fail(rc, why + " (the MPS state is kept at bond capacity " + std::to_string(old) + ")");
  }
  return DQ_OK;
}

int dq_mps_bond_dims(dq_mps_t h, uint32_t* dims) {
  clear_error();
  DQ_TRY(check_mps(h));
  if (!dims) return fail(DQ_ERR_INVALID_ARG, "null output");
  DeviceGuard g(h->device);
  DQ_CUDA_TRY(cudaMemcpyAsync(dims, h->dims, sizeof(uint32_t) * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
  DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DQ_OK;
}

int dq_mps_to_state(dq_mps_t h, dq_state_t out) {
  clear_error();
  DQ_TRY(check_mps(h));
  DQ_TRY(check_handle_lazy(out));
  if (out->n != h->n) return fail(DQ_ERR_INVALID_ARG, "the state must have the MPS's qubit count");
  if (out->device != h->device) return fail(DQ_ERR_INVALID_ARG, "the state must live on the MPS's device");
  DeviceGuard g(h->device);
  std::vector<uint32_t> dims(h->n + 1);
  DQ_CUDA_TRY(cudaMemcpyAsync(dims.data(), h->dims, sizeof(uint32_t) * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
  DQ_CUDA_TRY(cudaStreamSynchronize(h->stream));
  DQ_TRY(sync_stream(out));
  out->lazy_basis = -1;
  reset_perm(out);
  // W_k lives in `out` when n - 1 - k is even, else in tmp (both 2^n amplitudes)
  double2* tmp = nullptr;
  const size_t bytes = sizeof(double2) * (size_t)out->len;
  if (h->n > 1) DQ_CUDA_TRY(pool_malloc_async((void**)&tmp, bytes, h->stream));
  double2* one = nullptr;
  DQ_CUDA_TRY(pool_malloc_async((void**)&one, sizeof(double2), h->stream));
  const double2 o = make_double2(1.0, 0.0);
  cudaError_t e = cudaMemcpyAsync(one, &o, sizeof(o), cudaMemcpyHostToDevice, h->stream);
  const double2* w = one;
  for (uint32_t k = 0; k <= h->n; ++k)
    if (dims[k] == 0 || dims[k] > h->cap || (k < h->n && (2ull << k) * dims[k + 1] > out->len) ||
        ((k == 0 || k == h->n) && dims[k] != 1))
      e = cudaErrorInvalidValue;
  for (uint32_t k = 0; k < h->n && e == cudaSuccess; ++k) {
    double2* wn = ((h->n - 1 - k) % 2 == 0) ? out->amp : tmp;
    const uint64_t total = (2ull << k) * dims[k + 1];
    const unsigned grid = grid_for(total, 256, h->device);
    const double2* a = h->t + (uint64_t)k * h->batch * 2ull * h->cap * h->cap;
    k_mps_expand<<<grid, 256, 0, h->stream>>>(w, wn, a, k, dims[k], dims[k + 1], h->cap);
    e = cudaGetLastError();
    w = wn;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFreeAsync(one, h->stream);
  if (tmp) cudaFreeAsync(tmp, h->stream);
  cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(DQ_ERR_CUDA, std::string("MPS to_statevector: ") + cudaGetErrorString(e));
  return DQ_OK;
}

int dq_mps_run_shots(int device, uint32_t n, uint32_t max_bond, double truncation_threshold,
                     const dq_inst* prog, uint64_t ninst, const dq_cond* conds, uint64_t nconds,
                     uint64_t base_seed, uint64_t shot0, uint64_t shots, int32_t* cbits_out,
                     uint64_t ncbits, uint32_t batch, dq_mps_stats* stats) {
  clear_error();
  if ((ninst && !prog) || (nconds && !conds) || (shots && ncbits && !cbits_out))
    return fail(DQ_ERR_INVALID_ARG, "null program, condition or cbit buffer");
  if (ncbits > (1u << 26)) return fail(DQ_ERR_INVALID_ARG, "classical register array too large");
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->failed_inst = -1;
  }
  std::vector<MpsOp> ops;
  int64_t failed = -1;
  {
    int rc = lower(n, prog, ninst, conds, nconds, ncbits, ops, &failed);
    if (rc != DQ_OK) {
      if (stats) stats->failed_inst = failed;
      return rc;
    }
  }
  if (shots == 0) return DQ_OK;
  dq_mps_s* h = nullptr;
  DQ_TRY(new_handle(n, device, max_bond, truncation_threshold, &h));
  DeviceGuard g(device);
  const uint32_t bmax = batch ? batch : 4096u;
  // device memory for one batch: at most a quarter of the free memory
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const uint64_t budget = std::max<uint64_t>(free_b / 4, 1ull << 28);
  int rc = DQ_OK;
  double total_ms = 0.0;
  unsigned long long calls = 0;
  std::vector<uint64_t> seeds;
  for (uint64_t s0 = 0; s0 < shots && rc == DQ_OK;) {
    const uint64_t fit = std::max<uint64_t>(budget / replica_bytes(n, h->cap, 1), 1);
    const uint32_t nb = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(bmax, fit), shots - s0);
    seeds.resize(nb);
    for (uint32_t b = 0; b < nb; ++b) seeds[b] = base_seed + shot0 + s0 + b;  // wrapping
    int st = 0, fi = 0;
    double ms = 0.0;
    bool shrink = false;
    rc = run_batch(h, ops, conds, nconds, seeds.data(), nb, (uint32_t)ncbits, &st, &fi, &ms, budget,
                   &shrink);
    if (rc != DQ_OK) break;
    if (shrink) continue;  // capacity grew: redo this chunk with fewer replicas
    int64_t f64 = -1;
    rc = map_status(st, fi, &f64);
    if (rc != DQ_OK) {
      if (stats) stats->failed_inst = f64;
      break;
    }
    total_ms += ms;
    unsigned long long c = 0;
    cudaMemcpy(&c, h->svd_calls, sizeof(c), cudaMemcpyDeviceToHost);
    calls += c;
    if (ncbits) {
      const cudaError_t e = cudaMemcpy(cbits_out + s0 * ncbits, h->cbits, sizeof(int32_t) * ncbits * nb,
                                       cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, std::string("MPS cbits: ") + cudaGetErrorString(e));
    }
    s0 += nb;
  }
  if (stats) {
    stats->kernel_ms = total_ms;
    stats->svd_calls = calls;
    stats->capacity = h->cap;
    stats->replicas = h->batch;
  }
  destroy_handle(h);
  return rc;
}

}  // extern "C"
