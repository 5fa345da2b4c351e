// dq_gates.hpp — host-side gate matrices and their kernel classes.
//
// The matrices follow src/gates.rs:18-261 of the reference (row-major,
// qubits[0] = most significant bit of the row index) with the same libm
// calls and the same complex operation order (host code is built without
// FMA contraction), so the values match the Rust crate bit for bit.  The
// dispatcher mapping (which matrix and qubit order each instruction kind
// gets) follows statevector/simulator.rs:386-632.
//
// Every matrix is then classified into the cheapest kernel that reproduces
// the reference's dense arithmetic exactly:
//   ONE_Q   2x2 U on a target, optional all-ones controls (apply_one_qubit,
//           and the controlled gates cx..c4x whose dense rows reduce to it)
//   PHASE   diag(1, e) on a target with controls: only |1..1> amplitudes move
//   XPERM   X on a target with controls: a pure pair exchange
//   SWAP    exchange of |..01..> and |..10..> with controls (swap, cswap)
//   DIAG    general diagonal on k qubits (rzz, rc3x)
//   DENSE   anything else (rxx, psi+-, phi+): dense matvec, zero terms skipped
// Skipping a zero matrix entry only drops an addition of a signed zero, so
// every class is bit-identical to engine::apply_n_qubit up to the sign of
// exact zeros.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/dqsim_cuda.h"

namespace dq {

struct hc {  // host complex128 with num-complex operation order
  double re, im;
};
inline hc H(double re, double im) { return hc{re, im}; }
inline hc R(double re) { return hc{re, 0.0}; }
inline hc operator*(hc a, hc b) { return hc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline hc operator+(hc a, hc b) { return hc{a.re + b.re, a.im + b.im}; }
inline hc operator-(hc a) { return hc{-a.re, -a.im}; }
inline bool is_zero(hc a) { return a.re == 0.0 && a.im == 0.0; }
inline bool is_one(hc a) { return a.re == 1.0 && a.im == 0.0; }

enum GateClass { GC_NONE = 0, GC_ONE_Q, GC_PHASE, GC_XPERM, GC_SWAP, GC_DIAG, GC_DENSE };

struct Gate {
  uint32_t k = 0;           // number of qubits of the dense matrix
  uint32_t qubits[5] = {};  // qubits[0] = MSB of the matrix index
  hc m[32 * 32];            // row-major 2^k x 2^k
};

struct GateOp {             // a gate reduced to its kernel class
  GateClass cls = GC_NONE;
  uint32_t target = 0;      // ONE_Q / PHASE / XPERM
  uint32_t target2 = 0;     // SWAP: the two exchanged qubits are target, target2
  uint64_t ctrl_mask = 0;   // controls (all must be 1)
  hc u[4];                  // ONE_Q: 2x2; PHASE: u[0] = e
  Gate dense;               // DIAG / DENSE: full matrix (qubit order kept)
};

// ---- single-qubit matrices (gates.rs:18-84) -------------------------------
inline void u3_matrix(double theta, double phi, double lam, hc m[4]) {
  const double ct = cos(theta / 2.0), st = sin(theta / 2.0);
  m[0] = R(ct);
  m[1] = -(H(cos(lam), sin(lam)) * R(st));
  m[2] = H(cos(phi), sin(phi)) * R(st);
  m[3] = H(cos(phi + lam), sin(phi + lam)) * R(ct);
}

// Returns false if kind is not a one-qubit gate.
inline bool matrix_1q(int kind, const double* p, hc m[4]) {
  const double s = M_SQRT1_2;
  auto set = [&](hc a, hc b, hc c, hc d) { m[0] = a; m[1] = b; m[2] = c; m[3] = d; };
  switch (kind) {
    case DQ_ID: case DQ_U0: set(R(1), R(0), R(0), R(1)); return true;
    case DQ_X: set(R(0), R(1), R(1), R(0)); return true;
    case DQ_Y: set(R(0), H(0, -1), H(0, 1), R(0)); return true;
    case DQ_Z: set(R(1), R(0), R(0), R(-1)); return true;
    case DQ_H: set(R(s), R(s), R(s), R(-s)); return true;
    case DQ_S: set(R(1), R(0), R(0), H(0, 1)); return true;
    case DQ_SDG: set(R(1), R(0), R(0), H(0, -1)); return true;
    case DQ_T: set(R(1), R(0), R(0), H(s, s)); return true;
    case DQ_TDG: set(R(1), R(0), R(0), H(s, -s)); return true;
    case DQ_SX: set(H(0.5, 0.5), H(0.5, -0.5), H(0.5, -0.5), H(0.5, 0.5)); return true;
    case DQ_SXDG: set(H(0.5, -0.5), H(0.5, 0.5), H(0.5, 0.5), H(0.5, -0.5)); return true;
    case DQ_U3: case DQ_U: u3_matrix(p[0], p[1], p[2], m); return true;
    case DQ_U2: u3_matrix(M_PI / 2.0, p[0], p[1], m); return true;
    case DQ_U1: case DQ_P: set(R(1), R(0), R(0), H(cos(p[0]), sin(p[0]))); return true;
    case DQ_RX: {
      const double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      set(R(c2), H(0, -s2), H(0, -s2), R(c2));
      return true;
    }
    case DQ_RY: {
      const double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      set(R(c2), R(-s2), R(s2), R(c2));
      return true;
    }
    case DQ_RZ: {
      const double phi = p[0];
      set(H(cos(-phi / 2.0), sin(-phi / 2.0)), R(0), R(0), H(cos(phi / 2.0), sin(phi / 2.0)));
      return true;
    }
    default: return false;
  }
}

inline bool is_one_qubit_kind(int kind) {
  return (kind >= DQ_ID && kind <= DQ_U0);
}

// ---- multi-qubit matrices (gates.rs:90-261, simulator.rs:465-590) ---------
inline void identity(hc* m, uint32_t dim) {
  for (uint32_t i = 0; i < dim * dim; ++i) m[i] = R(0);
  for (uint32_t i = 0; i < dim; ++i) m[i * dim + i] = R(1);
}
inline void controlled_of(const hc u[4], hc m[16]) {
  identity(m, 4);
  m[10] = u[0]; m[11] = u[1]; m[14] = u[2]; m[15] = u[3];
}

// Fills g for a multi-qubit kind; returns false if kind is not such a gate.
inline bool matrix_nq(const dq_inst& in, Gate& g) {
  const double s = M_SQRT1_2;
  hc* m = g.m;
  hc u[4];
  for (int i = 0; i < in.nq && i < 5; ++i) g.qubits[i] = (uint32_t)in.q[i];
  switch (in.kind) {
    case DQ_CX: case DQ_G_CX:
      identity(m, 4); m[10] = R(0); m[15] = R(0); m[11] = R(1); m[14] = R(1); g.k = 2; return true;
    case DQ_CZ: case DQ_G_CZ:
      identity(m, 4); m[15] = R(-1); g.k = 2; return true;
    case DQ_CY:
      identity(m, 4); m[10] = R(0); m[15] = R(0); m[11] = H(0, -1); m[14] = H(0, 1); g.k = 2; return true;
    case DQ_CH:
      identity(m, 4); m[10] = R(s); m[11] = R(s); m[14] = R(s); m[15] = R(-s); g.k = 2; return true;
    case DQ_SWAP:
      identity(m, 4); m[5] = R(0); m[10] = R(0); m[6] = R(1); m[9] = R(1); g.k = 2; return true;
    case DQ_CSX:
      identity(m, 4);
      m[10] = H(0.5, 0.5); m[11] = H(0.5, -0.5); m[14] = H(0.5, -0.5); m[15] = H(0.5, 0.5);
      g.k = 2; return true;
    case DQ_CRX: matrix_1q(DQ_RX, in.p, u); controlled_of(u, m); g.k = 2; return true;
    case DQ_CRY: matrix_1q(DQ_RY, in.p, u); controlled_of(u, m); g.k = 2; return true;
    case DQ_CRZ: matrix_1q(DQ_RZ, in.p, u); controlled_of(u, m); g.k = 2; return true;
    case DQ_CU1: case DQ_CP: matrix_1q(DQ_U1, in.p, u); controlled_of(u, m); g.k = 2; return true;
    case DQ_CU3: u3_matrix(in.p[0], in.p[1], in.p[2], u); controlled_of(u, m); g.k = 2; return true;
    case DQ_CU: {
      hc inner[4];
      const hc phase = H(cos(in.p[3]), sin(in.p[3]));
      u3_matrix(in.p[0], in.p[1], in.p[2], inner);
      for (int i = 0; i < 4; ++i) u[i] = phase * inner[i];
      controlled_of(u, m);
      g.k = 2;
      return true;
    }
    case DQ_RXX: {
      const double cv = cos(in.p[0] / 2.0), sv = sin(in.p[0] / 2.0);
      for (int i = 0; i < 16; ++i) m[i] = R(0);
      m[0] = R(cv); m[3] = H(0, -sv); m[5] = R(cv); m[6] = H(0, -sv);
      m[9] = H(0, -sv); m[10] = R(cv); m[12] = H(0, -sv); m[15] = R(cv);
      g.k = 2;
      return true;
    }
    case DQ_RZZ: {
      const double h2 = in.p[0] / 2.0;
      const hc ep = H(cos(h2), sin(h2)), em = H(cos(h2), -sin(h2));
      for (int i = 0; i < 16; ++i) m[i] = R(0);
      m[0] = em; m[5] = ep; m[10] = ep; m[15] = em;
      g.k = 2;
      return true;
    }
    case DQ_G_PSI_MINUS: case DQ_G_PSI_PLUS: {
      const double pm[16] = {0, s, 0, s, s, 0, s, 0, -s, 0, s, 0, 0, -s, 0, s};
      for (int i = 0; i < 16; ++i) m[i] = R(pm[i]);
      if (in.kind == DQ_G_PSI_PLUS)
        for (int i = 8; i < 16; ++i) m[i] = -m[i];
      g.k = 2;
      return true;
    }
    case DQ_G_PHI_PLUS: {
      const double pp[16] = {s, 0, s, 0, 0, s, 0, s, 0, s, 0, -s, s, 0, -s, 0};
      for (int i = 0; i < 16; ++i) m[i] = R(pp[i]);
      g.k = 2;
      return true;
    }
    case DQ_CCX:
      identity(m, 8); m[54] = R(0); m[63] = R(0); m[55] = R(1); m[62] = R(1); g.k = 3; return true;
    case DQ_CSWAP:
      identity(m, 8); m[45] = R(0); m[54] = R(0); m[46] = R(1); m[53] = R(1); g.k = 3; return true;
    case DQ_RCCX:
      identity(m, 8); m[54] = R(0); m[63] = R(0); m[55] = H(0, 1); m[62] = H(0, -1); g.k = 3; return true;
    case DQ_RC3X:
      identity(m, 16); m[14 * 16 + 14] = H(0, 1); m[14 * 16 + 15] = R(0); m[15 * 16 + 14] = R(0);
      m[15 * 16 + 15] = H(0, -1); g.k = 4; return true;
    case DQ_C3X:
      identity(m, 16); m[14 * 16 + 14] = R(0); m[15 * 16 + 15] = R(0); m[14 * 16 + 15] = R(1);
      m[15 * 16 + 14] = R(1); g.k = 4; return true;
    case DQ_C3SQRTX:
      identity(m, 16);
      m[14 * 16 + 14] = H(0.5, 0.5); m[14 * 16 + 15] = H(0.5, -0.5);
      m[15 * 16 + 14] = H(0.5, -0.5); m[15 * 16 + 15] = H(0.5, 0.5);
      g.k = 4; return true;
    case DQ_C4X:
      identity(m, 32); m[30 * 32 + 30] = R(0); m[31 * 32 + 31] = R(0); m[30 * 32 + 31] = R(1);
      m[31 * 32 + 30] = R(1); g.k = 5; return true;
    default:
      return false;
  }
}

// Reduce a 2x2 (with controls) to PHASE / XPERM / ONE_Q.
inline void classify_1q(const hc u[4], uint32_t target, uint64_t ctrl, GateOp& op) {
  op.target = target;
  op.ctrl_mask = ctrl;
  if (is_one(u[0]) && is_zero(u[1]) && is_zero(u[2])) {
    op.cls = GC_PHASE;
    op.u[0] = u[3];
    return;
  }
  if (is_zero(u[0]) && is_zero(u[3]) && is_one(u[1]) && is_one(u[2])) {
    op.cls = GC_XPERM;
    return;
  }
  op.cls = GC_ONE_Q;
  for (int i = 0; i < 4; ++i) op.u[i] = u[i];
}

// Classify a dense gate into its cheapest exact kernel class.
inline void classify(const Gate& g, GateOp& op) {
  const uint32_t k = g.k, dim = 1u << k;
  const hc* m = g.m;
  // controlled-1q: identity except the bottom-right 2x2 block
  bool ctl = true;
  for (uint32_t r = 0; r < dim && ctl; ++r)
    for (uint32_t c = 0; c < dim; ++c) {
      if (r >= dim - 2 && c >= dim - 2) continue;
      const hc v = m[r * dim + c];
      if (r == c ? !is_one(v) : !is_zero(v)) { ctl = false; break; }
    }
  if (ctl) {
    uint64_t cm = 0;
    for (uint32_t b = 0; b + 1 < k; ++b) cm |= 1ULL << g.qubits[b];
    const hc u[4] = {m[(dim - 2) * dim + dim - 2], m[(dim - 2) * dim + dim - 1],
                     m[(dim - 1) * dim + dim - 2], m[(dim - 1) * dim + dim - 1]};
    classify_1q(u, g.qubits[k - 1], cm, op);
    return;
  }
  // controlled swap of the two least-significant gate qubits
  if (k >= 2) {
    bool sw = true;
    const uint32_t r01 = dim - 3, r10 = dim - 2;  // ...01 and ...10 with controls set
    for (uint32_t r = 0; r < dim && sw; ++r)
      for (uint32_t c = 0; c < dim; ++c) {
        const hc v = m[r * dim + c];
        bool want_one;
        if (r == r01) want_one = (c == r10);
        else if (r == r10) want_one = (c == r01);
        else want_one = (r == c);
        if (want_one ? !is_one(v) : !is_zero(v)) { sw = false; break; }
      }
    if (sw) {
      uint64_t cm = 0;
      for (uint32_t b = 0; b + 2 < k; ++b) cm |= 1ULL << g.qubits[b];
      op.cls = GC_SWAP;
      op.target = g.qubits[k - 2];
      op.target2 = g.qubits[k - 1];
      op.ctrl_mask = cm;
      return;
    }
  }
  bool diag = true;
  for (uint32_t r = 0; r < dim && diag; ++r)
    for (uint32_t c = 0; c < dim; ++c)
      if (r != c && !is_zero(m[r * dim + c])) { diag = false; break; }
  op.cls = diag ? GC_DIAG : GC_DENSE;
  op.dense = g;
}

// ---- fuse_circuit (types.rs:239-293) ------------------------------------------
// One simulate_shots trajectory runs the fused program: consecutive
// unconditional single-qubit gates on a qubit are multiplied into one 2x2
// (new = gate * pending), a pending matrix is flushed right before the first
// non-fusable instruction touching its qubit, matrices within 1e-10 of the
// identity are dropped, and the rest are flushed at the end (ascending qubit
// order; the reference iterates a HashMap there, which only affects the
// discarded final state).
struct FusedEntry {
  int64_t inst;  // >= 0: original instruction index; -1: fused 2x2 below
  uint32_t qubit;
  hc m[4];
};

inline void matmul2(const hc a[4], const hc b[4], hc out[4]) {
  const hc r0 = a[0] * b[0] + a[1] * b[2];
  const hc r1 = a[0] * b[1] + a[1] * b[3];
  const hc r2 = a[2] * b[0] + a[3] * b[2];
  const hc r3 = a[2] * b[1] + a[3] * b[3];
  out[0] = r0; out[1] = r1; out[2] = r2; out[3] = r3;
}

inline bool near_identity(const hc m[4]) {
  return hypot(m[0].re - 1.0, m[0].im) < 1e-10 && hypot(m[1].re, m[1].im) < 1e-10 &&
         hypot(m[2].re, m[2].im) < 1e-10 && hypot(m[3].re - 1.0, m[3].im) < 1e-10;
}

inline std::vector<FusedEntry> fuse_program(const dq_inst* prog, uint64_t ninst, uint32_t n) {
  std::vector<FusedEntry> out;
  out.reserve(ninst + n);
  std::vector<hc> pend(4 * (size_t)(n ? n : 1));
  std::vector<char> has(n ? n : 1, 0);
  auto flush = [&](uint32_t q) {
    if (q >= n || !has[q]) return;
    has[q] = 0;
    if (near_identity(&pend[4 * q])) return;
    FusedEntry e;
    e.inst = -1;
    e.qubit = q;
    for (int i = 0; i < 4; ++i) e.m[i] = pend[4 * q + i];
    out.push_back(e);
  };
  for (uint64_t i = 0; i < ninst; ++i) {
    const dq_inst& in = prog[i];
    hc m[4];
    if (in.cond_count == 0 && matrix_1q(in.kind, in.p, m)) {
      const uint32_t q = (uint32_t)in.q[0];
      if (!has[q]) {
        has[q] = 1;
        pend[4 * q] = R(1); pend[4 * q + 1] = R(0); pend[4 * q + 2] = R(0); pend[4 * q + 3] = R(1);
      }
      matmul2(m, &pend[4 * q], &pend[4 * q]);
      continue;
    }
    if (in.kind != DQ_BARRIER && in.kind != DQ_CLASSICAL)
      for (int t = 0; t < in.nq && t < DQ_MAX_INST_QUBITS; ++t)
        if (in.q[t] >= 0) flush((uint32_t)in.q[t]);
    FusedEntry e;
    e.inst = (int64_t)i;
    e.qubit = 0;
    out.push_back(e);
  }
  for (uint32_t q = 0; q < n; ++q) flush(q);
  return out;
}

}  // namespace dq
