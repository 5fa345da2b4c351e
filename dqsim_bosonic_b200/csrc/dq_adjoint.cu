// dq_adjoint.cu — Pauli-sum observables and adjoint differentiation.
//
// No counterpart in the reference engine (src/engine.rs has no gradients);
// the state layout, gate matrices (dq_gates.hpp, after src/gates.rs) and the
// forward pass (dq_run) are the engine's own.
//
// Adjoint method.  For psi_k = U_k ... U_1 psi_0 and E = <psi_P|H|psi_P>,
//   dE/dtheta = 2 Re <lambda_k| dU_k/dtheta |psi_{k-1}>,
//   lambda_P = H psi_P,  lambda_{k-1} = U_k^dagger lambda_k.
// The backward pass holds psi and lambda in HBM and walks the program in
// reverse; one kernel per parametrised gate reads (psi_k, lambda_k), writes
// (psi_{k-1}, lambda_{k-1}) and reduces the gradient terms of all the gate's
// parameters in the same pass: 64 B per amplitude per gate, no stored
// intermediate states.  Gates without a differentiated parameter are undone
// with the exact per-gate kernels (one launch per vector).
//
// Observables.  H = sum_t c_t P_t with P_t = i^{ny} X^{x_t} Z^{z_t}, so
//   (P_t psi)[j] = i^{ny} (-1)^{popcount((j ^ x_t) & z_t)} psi[j ^ x_t].
// Terms are grouped by x mask; k_pauli gathers psi[j ^ x] once per group.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "dq_adjsweep.cuh"
#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_fused.cuh"
#include "dq_gates.hpp"
#include "dq_handle.cuh"
#include "dq_reduce.cuh"

namespace dq {
namespace {

constexpr uint64_t kMaxTerms = 65536;

struct PauliGroup {  // device layout
  uint64_t x;
  uint32_t first, count;
};
struct PauliTerm {  // device layout: complex coefficient c * i^ny and z mask
  double cre, cim;
  uint64_t z;
  uint64_t pad;
};

__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}

// lambda = H psi (when STORE) and E = Re <psi|H psi>.
template <bool STORE>
__device__ __forceinline__ void pauli_body(const double2* __restrict__ psi, double2* __restrict__ lam,
                                           uint64_t len, const PauliGroup* __restrict__ groups,
                                           uint32_t ngroups, const PauliTerm* __restrict__ terms,
                                           double* partial, unsigned* counter, double* out) {
  double e = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < len; j += stride) {
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t g = 0; g < ngroups; ++g) {
      const uint64_t x = __ldg(&groups[g].x);
      const uint32_t f = __ldg(&groups[g].first), c = __ldg(&groups[g].count);
      const uint64_t src = j ^ x;
      double2 coef = make_double2(0.0, 0.0);
      for (uint32_t t = f; t < f + c; ++t) {
        const double cr = __ldg(&terms[t].cre), ci = __ldg(&terms[t].cim);
        const bool neg = __popcll(src & __ldg(&terms[t].z)) & 1;
        coef.x += neg ? -cr : cr;
        coef.y += neg ? -ci : ci;
      }
      acc = cfma(coef, psi[src], acc);
    }
    if (STORE) lam[j] = acc;
    const double2 p = psi[j];
    e = fma(p.x, acc.x, fma(p.y, acc.y, e));
  }
  double v[1] = {e};
  finish_partials<1>(v, partial, counter, out);
}

template <bool STORE>
__global__ void k_pauli(const double2* __restrict__ psi, double2* __restrict__ lam, uint64_t len,
                        const PauliGroup* __restrict__ groups, uint32_t ngroups,
                        const PauliTerm* __restrict__ terms, double* partial, unsigned* counter,
                        double* out) {
  pauli_body<STORE>(psi, lam, len, groups, ngroups, terms, partial, counter, out);
}

// The same for B states in one launch: state b (blockIdx.y) at psi + b len,
// its lambda at lam + b len, its reduction scratch at partial + b gridDim.x
// and counter + b, its expectation value at out[b * out_stride].
__global__ void k_pauli_multi(const double2* __restrict__ psi, double2* __restrict__ lam,
                              uint64_t len, const PauliGroup* __restrict__ groups, uint32_t ngroups,
                              const PauliTerm* __restrict__ terms, double* partial,
                              unsigned* counter, double* out, uint64_t out_stride) {
  const uint64_t b = blockIdx.y;
  pauli_body<true>(psi + b * len, lam + b * len, len, groups, ngroups, terms,
                   partial + b * gridDim.x, counter + b, out + b * out_stride);
}

// One parametrised 2x2 gate (controls: all set) on psi and lambda.
struct Adj1Args {
  double2 v[4];      // U^dagger
  double2 d[4][4];   // dU/dtheta_j, j < np
  uint32_t pos[9];   // ascending zero-insertion positions (target + controls)
  int npos;
  uint32_t target;
  uint64_t cmask;
};

template <int NP>
__global__ void __launch_bounds__(kRedThreads) k_adj_1q(double2* __restrict__ psi,
                                                        double2* __restrict__ lam, uint64_t count,
                                                        const Adj1Args a, double* partial,
                                                        unsigned* counter, double* out) {
  double acc[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) acc[j] = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tb = 1ULL << a.target;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += stride) {
    const uint64_t i0 = insert_zeros(k, a.pos, a.npos) | a.cmask, i1 = i0 | tb;
    const double2 a0 = psi[i0], a1 = psi[i1], b0 = lam[i0], b1 = lam[i1];
    const double2 p0 = cfma(a.v[1], a1, cmul_f(a.v[0], a0));
    const double2 p1 = cfma(a.v[3], a1, cmul_f(a.v[2], a0));
    psi[i0] = p0;
    psi[i1] = p1;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const double2 w0 = cfma(a.d[j][1], p1, cmul_f(a.d[j][0], p0));
      const double2 w1 = cfma(a.d[j][3], p1, cmul_f(a.d[j][2], p0));
      acc[j] = fma(b0.x, w0.x, fma(b0.y, w0.y, fma(b1.x, w1.x, fma(b1.y, w1.y, acc[j]))));
    }
    lam[i0] = cfma(a.v[1], b1, cmul_f(a.v[0], b0));
    lam[i1] = cfma(a.v[3], b1, cmul_f(a.v[2], b0));
  }
  finish_partials<NP>(acc, partial, counter, out);
}

// One parametrised dense two-qubit gate (rxx, rzz): qa = MSB of the 4x4 index.
struct Adj2Args {
  double2 v[16];
  double2 d[16];
  uint32_t pos[2];
  uint32_t qa, qb;
};

__global__ void __launch_bounds__(kRedThreads) k_adj_2q(double2* __restrict__ psi,
                                                        double2* __restrict__ lam, uint64_t count,
                                                        const Adj2Args a, double* partial,
                                                        unsigned* counter, double* out) {
  double acc = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t ba = 1ULL << a.qa, bb = 1ULL << a.qb;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += stride) {
    const uint64_t base = insert_zeros(k, a.pos, 2);
    const uint64_t idx[4] = {base, base | bb, base | ba, base | ba | bb};
    double2 x[4], y[4], p[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      x[r] = psi[idx[r]];
      y[r] = lam[idx[r]];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 4; ++c) s = cfma(a.v[r * 4 + c], x[c], s);
      p[r] = s;
      psi[idx[r]] = s;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double2 w = make_double2(0.0, 0.0), s = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        w = cfma(a.d[r * 4 + c], p[c], w);
        s = cfma(a.v[r * 4 + c], y[c], s);
      }
      acc = fma(y[r].x, w.x, fma(y[r].y, w.y, acc));
      lam[idx[r]] = s;
    }
  }
  double v[1] = {acc};
  finish_partials<1>(v, partial, counter, out);
}

// ---- host side ----------------------------------------------------------------------

inline double2 d2(hc z) { return make_double2(z.re, z.im); }
inline hc cj(hc z) { return hc{z.re, -z.im}; }
inline hc sc(hc z, double f) { return hc{z.re * f, z.im * f}; }
inline hc ei(double a) { return hc{cos(a), sin(a)}; }

// Number of angle parameters of a kind that adjoint differentiation covers.
int diff_param_count(int kind) {
  switch (kind) {
    case DQ_RX: case DQ_RY: case DQ_RZ: case DQ_U1: case DQ_P:
    case DQ_CRX: case DQ_CRY: case DQ_CRZ: case DQ_CU1: case DQ_CP:
    case DQ_RXX: case DQ_RZZ:
      return 1;
    case DQ_U2: return 2;
    case DQ_U3: case DQ_U: case DQ_CU3: return 3;
    case DQ_CU: return 4;
    default: return 0;
  }
}

// d u3(theta, phi, lam) / d(theta, phi, lam).
void u3_derivs(double th, double ph, double la, hc d[3][4]) {
  const double ct = cos(th / 2.0), st = sin(th / 2.0);
  const hc el = ei(la), ep = ei(ph), epl = ei(ph + la);
  d[0][0] = hc{-st / 2.0, 0.0};
  d[0][1] = sc(el, -ct / 2.0);
  d[0][2] = sc(ep, ct / 2.0);
  d[0][3] = sc(epl, -st / 2.0);
  const hc i1 = hc{0.0, 1.0};
  d[1][0] = hc{0, 0};
  d[1][1] = hc{0, 0};
  d[1][2] = i1 * sc(ep, st);
  d[1][3] = i1 * sc(epl, ct);
  d[2][0] = hc{0, 0};
  d[2][1] = i1 * sc(el, -st);
  d[2][2] = hc{0, 0};
  d[2][3] = i1 * sc(epl, ct);
}

// The 2x2 block u of a (controlled) one-qubit parametrised kind and its
// derivatives with respect to each parameter.
bool block_derivs(const dq_inst& in, hc u[4], hc d[4][4], int* np) {
  const double* p = in.p;
  *np = diff_param_count(in.kind);
  switch (in.kind) {
    case DQ_RX: case DQ_CRX: {
      matrix_1q(DQ_RX, p, u);
      const double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      d[0][0] = hc{-s2 / 2.0, 0}; d[0][1] = hc{0, -c2 / 2.0};
      d[0][2] = hc{0, -c2 / 2.0}; d[0][3] = hc{-s2 / 2.0, 0};
      return true;
    }
    case DQ_RY: case DQ_CRY: {
      matrix_1q(DQ_RY, p, u);
      const double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      d[0][0] = hc{-s2 / 2.0, 0}; d[0][1] = hc{-c2 / 2.0, 0};
      d[0][2] = hc{c2 / 2.0, 0}; d[0][3] = hc{-s2 / 2.0, 0};
      return true;
    }
    case DQ_RZ: case DQ_CRZ:
      matrix_1q(DQ_RZ, p, u);
      d[0][0] = hc{0, -0.5} * u[0]; d[0][1] = hc{0, 0};
      d[0][2] = hc{0, 0}; d[0][3] = hc{0, 0.5} * u[3];
      return true;
    case DQ_U1: case DQ_P: case DQ_CU1: case DQ_CP:
      matrix_1q(DQ_U1, p, u);
      d[0][0] = hc{0, 0}; d[0][1] = hc{0, 0}; d[0][2] = hc{0, 0};
      d[0][3] = hc{0, 1} * u[3];
      return true;
    case DQ_U2: {
      u3_matrix(M_PI / 2.0, p[0], p[1], u);
      hc t[3][4];
      u3_derivs(M_PI / 2.0, p[0], p[1], t);
      for (int i = 0; i < 4; ++i) { d[0][i] = t[1][i]; d[1][i] = t[2][i]; }
      return true;
    }
    case DQ_U3: case DQ_U: case DQ_CU3: {
      u3_matrix(p[0], p[1], p[2], u);
      hc t[3][4];
      u3_derivs(p[0], p[1], p[2], t);
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) d[j][i] = t[j][i];
      return true;
    }
    case DQ_CU: {
      hc inner[4], t[3][4];
      const hc g = ei(p[3]);
      u3_matrix(p[0], p[1], p[2], inner);
      u3_derivs(p[0], p[1], p[2], t);
      for (int i = 0; i < 4; ++i) u[i] = g * inner[i];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) d[j][i] = g * t[j][i];
      for (int i = 0; i < 4; ++i) d[3][i] = hc{0, 1} * u[i];
      return true;
    }
    default:
      return false;
  }
}

// The 4x4 of rxx / rzz and its derivative.
bool rxx_rzz_deriv(const dq_inst& in, hc m[16], hc dm[16]) {
  if (in.kind != DQ_RXX && in.kind != DQ_RZZ) return false;
  Gate g;
  matrix_nq(in, g);
  for (int i = 0; i < 16; ++i) {
    m[i] = g.m[i];
    dm[i] = hc{0, 0};
  }
  if (in.kind == DQ_RZZ) {
    dm[0] = hc{0, -0.5} * g.m[0];
    dm[5] = hc{0, 0.5} * g.m[5];
    dm[10] = hc{0, 0.5} * g.m[10];
    dm[15] = hc{0, -0.5} * g.m[15];
  } else {
    const double cv = cos(in.p[0] / 2.0), sv = sin(in.p[0] / 2.0);
    for (int i : {0, 5, 10, 15}) dm[i] = hc{-sv / 2.0, 0};
    for (int i : {3, 6, 9, 12}) dm[i] = hc{0, -cv / 2.0};
  }
  return true;
}

bool is_controlled_block(int kind) {
  switch (kind) {
    case DQ_CRX: case DQ_CRY: case DQ_CRZ: case DQ_CU1: case DQ_CP: case DQ_CU3: case DQ_CU:
      return true;
    default:
      return false;
  }
}

// The inverse of a gate instruction as a kernel-class op.
bool inverse_op(const dq_inst& in, GateOp& op) {
  hc u[4];
  if (matrix_1q(in.kind, in.p, u)) {
    const hc v[4] = {cj(u[0]), cj(u[2]), cj(u[1]), cj(u[3])};
    classify_1q(v, (uint32_t)in.q[0], 0, op);
    return true;
  }
  Gate g;
  if (!matrix_nq(in, g)) return false;
  const uint32_t dim = 1u << g.k;
  std::vector<hc> t(g.m, g.m + dim * dim);
  for (uint32_t r = 0; r < dim; ++r)
    for (uint32_t c = 0; c < dim; ++c) g.m[r * dim + c] = cj(t[c * dim + r]);
  classify(g, op);
  return true;
}

bool is_noop_kind(int kind) {
  return kind == DQ_ID || kind == DQ_U0 || kind == DQ_BARRIER || kind == DQ_CLASSICAL ||
         kind == DQ_G_NOOP;
}

// Validates a unitary program and its parameter map; counts differentiated slots.
int check_program_n(uint32_t n, const dq_inst* prog, uint64_t ninst, const int32_t* pidx,
                    uint64_t nparams, uint64_t* nslots) {
  if (ninst && !prog) return fail(DQ_ERR_INVALID_ARG, "null program");
  if (nparams && !pidx) return fail(DQ_ERR_INVALID_ARG, "null param_index with nparams > 0");
  if (nparams > (1ULL << 31)) return fail(DQ_ERR_INVALID_ARG, "too many parameters");
  uint64_t s = 0;
  for (uint64_t i = 0; i < ninst; ++i) {
    const dq_inst& in = prog[i];
    if (in.cond_count || in.kind == DQ_MEASURE || in.kind == DQ_RESET ||
        in.kind == DQ_G_OPAQUE || in.kind == DQ_G_UNSUPPORTED)
      return fail(DQ_ERR_UNSUPPORTED, "instruction " + std::to_string(i) +
                                          ": adjoint differentiation needs a unitary program "
                                          "(gates only, no measure/reset/conditions)");
    DQ_TRY(validate_inst(in, n, 0, 0, nullptr, i));
    if (!pidx) continue;
    const int np = diff_param_count(in.kind);
    for (int j = 0; j < 4; ++j) {
      const int32_t v = pidx[4 * i + j];
      if (v < -1 || (v >= 0 && (uint64_t)v >= nparams))
        return fail(DQ_ERR_INVALID_ARG, "instruction " + std::to_string(i) + ": param_index " +
                                            std::to_string(v) + " outside [-1, nparams)");
      if (v >= 0 && j >= np)
        return fail(DQ_ERR_INVALID_ARG, "instruction " + std::to_string(i) +
                                            ": parameter slot " + std::to_string(j) +
                                            " of this kind is not differentiable");
      if (v >= 0) ++s;
    }
  }
  *nslots = s;
  return DQ_OK;
}

int check_program(dq_state_t h, const dq_inst* prog, uint64_t ninst, const int32_t* pidx,
                  uint64_t nparams, uint64_t* nslots) {
  return check_program_n(h->n, prog, ninst, pidx, nparams, nslots);
}

struct DeviceTerms {
  PauliGroup* groups = nullptr;
  PauliTerm* terms = nullptr;
  uint32_t ngroups = 0;
};

int upload_terms(const dq_pauli_term* terms, uint64_t nterms, uint32_t n, cudaStream_t st,
                 DeviceTerms* out) {
  if (nterms && !terms) return fail(DQ_ERR_INVALID_ARG, "null terms");
  if (nterms > kMaxTerms) return fail(DQ_ERR_INVALID_ARG, "more than 65536 Pauli terms");
  const uint64_t reg = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
  std::vector<uint64_t> order(nterms);
  for (uint64_t t = 0; t < nterms; ++t) {
    if ((terms[t].xmask | terms[t].zmask) & ~reg)
      return fail(DQ_ERR_INVALID_ARG, "Pauli term " + std::to_string(t) + " acts outside the register");
    if (!std::isfinite(terms[t].coeff))
      return fail(DQ_ERR_INVALID_ARG, "Pauli term " + std::to_string(t) + " has a non-finite coefficient");
    order[t] = t;
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](uint64_t a, uint64_t b) { return terms[a].xmask < terms[b].xmask; });
  std::vector<PauliGroup> g;
  std::vector<PauliTerm> tv(nterms ? nterms : 1);
  for (uint64_t r = 0; r < nterms; ++r) {
    const dq_pauli_term& t = terms[order[r]];
    if (g.empty() || g.back().x != t.xmask) g.push_back(PauliGroup{t.xmask, (uint32_t)r, 0});
    ++g.back().count;
    const int ny = __builtin_popcountll(t.xmask & t.zmask) & 3;
    const double c = t.coeff;
    const double re[4] = {c, 0.0, -c, 0.0}, im[4] = {0.0, c, 0.0, -c};
    tv[r] = PauliTerm{re[ny], im[ny], t.zmask, 0};
  }
  if (g.empty()) g.push_back(PauliGroup{0, 0, 0});
  out->ngroups = (uint32_t)g.size();
  DQ_CUDA_TRY(pool_malloc_async((void**)&out->groups, sizeof(PauliGroup) * g.size(), st));
  DQ_CUDA_TRY(pool_malloc_async((void**)&out->terms, sizeof(PauliTerm) * tv.size(), st));
  DQ_CUDA_TRY(cudaMemcpyAsync(out->groups, g.data(), sizeof(PauliGroup) * g.size(),
                              cudaMemcpyHostToDevice, st));
  DQ_CUDA_TRY(cudaMemcpyAsync(out->terms, tv.data(), sizeof(PauliTerm) * tv.size(),
                              cudaMemcpyHostToDevice, st));
  // the host vectors go out of scope: make the copies complete first
  DQ_CUDA_TRY(cudaStreamSynchronize(st));
  return DQ_OK;
}

void free_terms(DeviceTerms& t, cudaStream_t st) {
  if (t.groups) cudaFreeAsync(t.groups, st);
  if (t.terms) cudaFreeAsync(t.terms, st);
  t.groups = nullptr;
  t.terms = nullptr;
}

int launch_pauli(dq_state_t h, double2* lam, const DeviceTerms& t, double* d_out) {
  const unsigned blocks = reduction_blocks(h->len, h->device);
  if (lam)
    k_pauli<true><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, h->len, t.groups, t.ngroups,
                                                         t.terms, h->sc.d_partial,
                                                         h->sc.d_counter, d_out);
  else
    k_pauli<false><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, nullptr, h->len, t.groups,
                                                          t.ngroups, t.terms, h->sc.d_partial,
                                                          h->sc.d_counter, d_out);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

// One backward step for a gate with differentiated slots; results (without
// the factor 2) go to d_out[0..np).
int launch_adj(dq_state_t h, double2* lam, const dq_inst& in, double* d_out) {
  hc u[4], d[4][4];
  int np = 0;
  if (block_derivs(in, u, d, &np)) {
    Adj1Args a{};
    a.v[0] = d2(cj(u[0])); a.v[1] = d2(cj(u[2]));
    a.v[2] = d2(cj(u[1])); a.v[3] = d2(cj(u[3]));
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < 4; ++i) a.d[j][i] = d2(d[j][i]);
    const bool ctl = is_controlled_block(in.kind);
    a.target = (uint32_t)(ctl ? in.q[1] : in.q[0]);
    a.cmask = ctl ? (1ULL << in.q[0]) : 0ULL;
    a.npos = 0;
    a.pos[a.npos++] = a.target;
    if (ctl) a.pos[a.npos++] = (uint32_t)in.q[0];
    std::sort(a.pos, a.pos + a.npos);
    const uint64_t count = h->len >> a.npos;
    const unsigned blocks = reduction_blocks(count, h->device);
    double* part = h->sc.d_partial;
    unsigned* ctr = h->sc.d_counter;
    switch (np) {
      case 1: k_adj_1q<1><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, count, a, part, ctr, d_out); break;
      case 2: k_adj_1q<2><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, count, a, part, ctr, d_out); break;
      case 3: k_adj_1q<3><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, count, a, part, ctr, d_out); break;
      case 4: k_adj_1q<4><<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, count, a, part, ctr, d_out); break;
      default: return fail(DQ_ERR_INTERNAL, "bad parameter count");
    }
    DQ_CUDA_TRY(cudaGetLastError());
    return DQ_OK;
  }
  Gate g;
  hc dm[16];
  if (!rxx_rzz_deriv(in, g.m, dm)) return fail(DQ_ERR_INTERNAL, "kind without derivative");
  Adj2Args a{};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      a.v[r * 4 + c] = d2(cj(g.m[c * 4 + r]));
      a.d[r * 4 + c] = d2(dm[r * 4 + c]);
    }
  a.qa = (uint32_t)in.q[0];
  a.qb = (uint32_t)in.q[1];
  a.pos[0] = std::min(a.qa, a.qb);
  a.pos[1] = std::max(a.qa, a.qb);
  const uint64_t count = h->len >> 2;
  const unsigned blocks = reduction_blocks(count, h->device);
  k_adj_2q<<<blocks, kRedThreads, 0, h->stream>>>(h->amp, lam, count, a, h->sc.d_partial,
                                                   h->sc.d_counter, d_out);
  DQ_CUDA_TRY(cudaGetLastError());
  return DQ_OK;
}

}  // namespace

bool adjoint_block_derivs(const dq_inst& in, hc u[4], hc d[4][4], int* np) {
  return block_derivs(in, u, d, np);
}
bool adjoint_rxx_rzz_deriv(const dq_inst& in, hc m[16], hc dm[16]) { return rxx_rzz_deriv(in, m, dm); }
bool adjoint_controlled_block(int kind) { return is_controlled_block(kind); }

}  // namespace dq

using namespace dq;

extern "C" {

int dq_expval_pauli(dq_state_t h, const dq_pauli_term* terms, uint64_t nterms, double* out) {
  DQ_TRY(check_handle(h));
  if (!out) return fail(DQ_ERR_INVALID_ARG, "null output");
  DeviceGuard g(h->device);
  DQ_TRY(canonicalize(h));
  DeviceTerms t;
  int rc = upload_terms(terms, nterms, h->n, h->stream, &t);
  double* d = h->sc.d_partial + kPartials - 1;
  if (rc == DQ_OK) rc = launch_pauli(h, nullptr, t, d);
  double v = 0.0;
  if (rc == DQ_OK) rc = read_scalars(h, d, 1, &v);
  free_terms(t, h->stream);
  DQ_TRY(rc);
  *out = v;
  return sync_stream(h);
}

int dq_adjoint(dq_state_t h, const dq_inst* prog, uint64_t ninst, const int32_t* param_index,
               uint64_t nparams, const dq_pauli_term* terms, uint64_t nterms,
               const dq_run_opts* opts, double* expval, double* grad, double* phase_ms) {
  DQ_TRY(check_handle_lazy(h));  // the forward dq_run starts from a lazy basis state
  if (!expval || (nparams && !grad)) return fail(DQ_ERR_INVALID_ARG, "null output");
  uint64_t nslots = 0;
  DQ_TRY(check_program(h, prog, ninst, param_index, nparams, &nslots));
  dq_run_opts o{};
  o.exec = DQ_EXEC_FUSED;
  if (opts) o = *opts;
  if (o.semantics != DQ_SEM_SIMULATE)
    return fail(DQ_ERR_INVALID_ARG, "dq_adjoint runs with DQ_SEM_SIMULATE semantics");
  o.profile = 0;
  DeviceGuard g(h->device);
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (phase_ms)
    for (auto& e : ev) DQ_CUDA_TRY(cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } evg{ev};
  auto mark = [&](int i) {
    if (ev[i]) cudaEventRecord(ev[i], h->stream);
  };

  // The observable's terms, lambda and the gradient slots are set up before
  // the forward pass (the term upload waits for the stream, an allocation
  // may block the host), so forward pass, lambda = H psi and backward pass
  // run back to back on the stream.
  DeviceTerms t;
  DQ_TRY(upload_terms(terms, nterms, h->n, h->stream, &t));
  void* lam_v = nullptr;
  int rc = cache_alloc(h->device, h->bytes, &lam_v);
  double2* lam = (double2*)lam_v;
  double* slots = nullptr;
  if (rc == DQ_OK) {
    cudaError_t e = pool_malloc_async((void**)&slots, sizeof(double) * (nslots + 1), h->stream);
    if (e != cudaSuccess) rc = fail(DQ_ERR_OOM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  }

  // forward pass
  mark(0);
  if (rc == DQ_OK) rc = dq_run(h, prog, ninst, nullptr, 0, 0, nullptr, 0, &o, nullptr);
  if (rc == DQ_OK) rc = canonicalize(h);
  mark(1);
  if (rc == DQ_OK) rc = launch_pauli(h, lam, t, slots + nslots);
  mark(2);

  // backward pass: slots are numbered in program order
  const bool fused_back = o.exec == DQ_EXEC_FUSED;
  AdjSweepStats ss;
  if (fused_back && rc == DQ_OK)
    rc = adjoint_backward_fused(h->amp, lam, h->n, prog, ninst, param_index, nslots, slots,
                                h->stream, h->device, &ss);
  uint64_t slot = nslots;
  for (uint64_t r = ninst; !fused_back && rc == DQ_OK && r-- > 0;) {
    const dq_inst& in = prog[r];
    if (is_noop_kind(in.kind)) continue;
    int nd = 0;
    if (param_index)
      for (int j = 0; j < 4; ++j) nd += param_index[4 * r + j] >= 0;
    if (nd > 0) {
      const int np = diff_param_count(in.kind);
      slot -= nd;
      // every parameter of the gate is reduced; unused slots land in a
      // scratch double past the end of the real ones
      double* tmp = h->sc.d_partial + kPartials - 8;
      rc = launch_adj(h, lam, in, np == nd && np > 0 ? slots + slot : tmp);
      if (rc == DQ_OK && !(np == nd)) {
        // scatter the differentiated subset from the scratch results
        int k = 0;
        for (int j = 0; j < np && rc == DQ_OK; ++j)
          if (param_index[4 * r + j] >= 0) {
            cudaError_t e = cudaMemcpyAsync(slots + slot + k, tmp + j, sizeof(double),
                                            cudaMemcpyDeviceToDevice, h->stream);
            if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
            ++k;
          }
      }
    } else {
      GateOp op;
      if (!inverse_op(in, op)) {
        rc = fail(DQ_ERR_INTERNAL, "instruction kind without a matrix");
        break;
      }
      rc = launch_gate(h->amp, h->n, op, h->stream, h->device, nullptr);
      if (rc == DQ_OK) rc = launch_gate(lam, h->n, op, h->stream, h->device, nullptr);
    }
  }

  mark(3);
  std::vector<double> host(nslots + 1, 0.0);
  if (rc == DQ_OK) {
    cudaError_t e = cudaMemcpyAsync(host.data(), slots, sizeof(double) * (nslots + 1),
                                    cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, cudaGetErrorString(e));
  }
  if (rc == DQ_OK) rc = sync_stream(h);
  if (slots) cudaFreeAsync(slots, h->stream);
  free_terms(t, h->stream);
  if (lam) {
    cudaStreamSynchronize(h->stream);
    cache_free(h->device, h->bytes, lam);
  }
  DQ_TRY(rc);
  if (phase_ms)
    for (int i = 0; i < 3; ++i) {
      float ms = 0.f;
      DQ_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      phase_ms[i] = ms;
    }
  if (phase_ms) phase_ms[3] = (double)ss.sweeps;
  *expval = host[nslots];
  for (uint64_t p = 0; p < nparams; ++p) grad[p] = 0.0;
  uint64_t s = 0;
  for (uint64_t i = 0; i < ninst; ++i) {
    if (!param_index || is_noop_kind(prog[i].kind)) continue;
    for (int j = 0; j < 4; ++j) {
      const int32_t v = param_index[4 * i + j];
      if (v >= 0) grad[v] += 2.0 * host[s++];
    }
  }
  return DQ_OK;
}


int dq_adjoint_batch(int device, uint32_t n, const dq_inst* prog, uint64_t ninst,
                     const int32_t* param_index, uint64_t nparams, const double* values,
                     uint64_t nsets, const dq_pauli_term* terms, uint64_t nterms, double* expvals,
                     double* grads, dq_adjoint_batch_stats* stats) {
  dq_adjoint_batch_stats acc{};
  if (stats) *stats = acc;
  if (n < 1 || n > kMaxQubits) return fail(DQ_ERR_INVALID_ARG, "nqubits must be in 1..34");
  uint64_t nslots = 0;
  DQ_TRY(check_program_n(n, prog, ninst, param_index, nparams, &nslots));
  if (nsets && (!expvals || (nparams && (!grads || !values))))
    return fail(DQ_ERR_INVALID_ARG, "null values or outputs");
  if (nsets == 0) return DQ_OK;
  int ndev = 0;
  DQ_TRY(dq_device_count(&ndev));
  if (device < 0 || device >= ndev) return fail(DQ_ERR_INVALID_ARG, "device index out of range");
  DeviceGuard g(device);
  const auto t0 = std::chrono::steady_clock::now();
  // DQSIM_ADJOINT_TIMING=1: host phase times on stderr
  static const bool timing = [] {
    const char* e = getenv("DQSIM_ADJOINT_TIMING");
    return e && atoi(e) != 0;
  }();
  auto tlast = t0;
  auto mark = [&](const char* what) {
    if (!timing) return;
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[dq_adjoint_batch] %-18s %8.3f ms\n", what,
            std::chrono::duration<double, std::milli>(now - tlast).count());
    tlast = now;
  };
  // each set's program: the parameter slots replaced by its values
  std::vector<std::vector<dq_inst>> progs(nsets);
  for (uint64_t s = 0; s < nsets; ++s) {
    progs[s].assign(prog, prog + ninst);
    if (!param_index) continue;
    for (uint64_t i = 0; i < ninst; ++i)
      for (int j = 0; j < 4; ++j) {
        const int32_t v = param_index[4 * i + j];
        if (v >= 0) progs[s][i].p[j] = values[s * nparams + (uint64_t)v];
      }
  }
  // plan every set on host threads: forward sweeps from |0...0>, backward sweeps
  struct SetPlan {
    std::vector<uint8_t> fblob;
    std::vector<uint64_t> foffs;
    uint32_t perm[64];
    int64_t synth = -1;
    uint32_t rb = 0;
    ABatchSet back;
    int rc = DQ_OK;
  };
  std::vector<SetPlan> plans(nsets);
  bool batched = n >= kFusedMinQubits;
  if (batched) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::min<uint64_t>(hw, nsets);
    auto work = [&](unsigned t) {
      for (uint64_t s = t; s < nsets; s += nt) {
        SetPlan& P = plans[s];
        for (uint32_t l = 0; l < 64; ++l) P.perm[l] = l;
        P.rc = fused_plan(n, progs[s].data(), ninst, DQ_SEM_SIMULATE, 7, 0, 0, &P.fblob, &P.foffs,
                          P.perm, &P.synth, &P.rb);
        if (P.rc == DQ_OK)
          P.rc = adjoint_backward_plan_set(n, progs[s].data(), ninst, param_index, nslots, &P.back);
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    uint32_t rb = 0;
    for (uint64_t s = 0; s < nsets; ++s)
      if (!plans[s].foffs.empty()) rb = plans[s].rb;
    for (uint64_t s = 0; s < nsets && batched; ++s)
      if (plans[s].rc != DQ_OK || plans[s].back.sweeps() == 0 ||
          (!plans[s].foffs.empty() && plans[s].rb != rb))
        batched = false;
    clear_error();
  }
  acc.plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  mark("programs+plan");
  if (!batched) {
    // set by set through dq_adjoint on one engine state
    dq_state_t h = nullptr;
    DQ_TRY(dq_state_create(n, device, &h));
    dq_run_opts o{};
    o.exec = DQ_EXEC_FUSED;
    int rc = DQ_OK;
    for (uint64_t s = 0; s < nsets && rc == DQ_OK; ++s) {
      rc = dq_state_reset(h);
      if (rc == DQ_OK)
        rc = dq_adjoint(h, progs[s].data(), ninst, param_index, nparams, terms, nterms, &o,
                        expvals + s, nparams ? grads + s * nparams : nullptr, nullptr);
    }
    dq_state_destroy(h);
    acc.groups = (uint32_t)nsets;
    if (stats) *stats = acc;
    return rc;
  }
  uint32_t rb = 0;
  for (uint64_t s = 0; s < nsets; ++s)
    if (!plans[s].foffs.empty()) rb = plans[s].rb;
  const uint64_t len = 1ULL << n;
  // sets resident at a time: psi and lambda of each in about half the free memory
  size_t freeb = 0, totalb = 0;
  DQ_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  const uint64_t per_set = 2 * sizeof(double2) * len + 64 * 1024;
  const uint64_t G = std::max<uint64_t>(1, std::min<uint64_t>(nsets, (freeb / 2) / per_set));
  cudaStream_t st = nullptr;
  DQ_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = DQ_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == DQ_OK) {
      cudaGetLastError();
      rc = fail(e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
    }
  };
  DeviceTerms t;
  rc = upload_terms(terms, nterms, n, st, &t);
  double2 *psi = nullptr, *lam = nullptr;
  double* slots = nullptr;
  double* part = nullptr;
  unsigned* ctr = nullptr;
  uint8_t* fblob = nullptr;
  SweepJob* d_jobs = nullptr;
  const unsigned pblocks = reduction_blocks(len, device);
  const uint64_t sl = nslots + 1;  // per set: gradient slots, then E
  // all forward programs in one device buffer, staged in pinned host memory
  // (recycled across calls) by host threads
  std::vector<uint64_t> fbase(nsets, 0);
  size_t fall_bytes = 0, kf = 0, kb = 0;
  for (uint64_t s = 0; s < nsets; ++s) {
    fbase[s] = fall_bytes;
    fall_bytes += (plans[s].fblob.size() + 15) / 16 * 16;
    kf = std::max(kf, plans[s].foffs.size());
    kb = std::max(kb, plans[s].back.sweeps());
  }
  fall_bytes = std::max<size_t>(fall_bytes, 16);
  struct PinnedStage {
    size_t bytes = 0;
    void* p = nullptr;
    ~PinnedStage() { pinned_free(bytes, p); }
  } fall;
  if (rc == DQ_OK) rc = pinned_alloc(fall_bytes, &fall.p);
  if (rc == DQ_OK) {
    fall.bytes = fall_bytes;
    uint8_t* dst = static_cast<uint8_t*>(fall.p);
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hw, nsets / 8 + 1));
    auto work = [&](unsigned t) {
      for (uint64_t s = t; s < nsets; s += nt)
        if (!plans[s].fblob.empty()) memcpy(dst + fbase[s], plans[s].fblob.data(), plans[s].fblob.size());
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
  }
  acc.forward_sweeps = kf;
  acc.backward_sweeps = kb;
  if (rc == DQ_OK) {
    // psi and lambda of the group come from the engine's size-keyed buffer
    // cache: repeated calls (an optimiser loop) do not pay cudaMalloc/cudaFree
    void* pv = nullptr;
    void* lv = nullptr;
    rc = cache_alloc(device, sizeof(double2) * len * G, &pv);
    if (rc == DQ_OK) rc = cache_alloc(device, sizeof(double2) * len * G, &lv);
    psi = (double2*)pv;
    lam = (double2*)lv;
    // the small buffers also from the cache: an optimiser loop repeats their sizes
    void* p = nullptr;
    if (rc == DQ_OK && (rc = cache_alloc(device, sizeof(double) * sl * G, &p)) == DQ_OK) slots = (double*)p;
    if (rc == DQ_OK && (rc = cache_alloc(device, sizeof(double) * pblocks * G, &p)) == DQ_OK) part = (double*)p;
    if (rc == DQ_OK && (rc = cache_alloc(device, sizeof(unsigned) * G, &p)) == DQ_OK) ctr = (unsigned*)p;
    if (rc == DQ_OK && (rc = cache_alloc(device, fall_bytes, &p)) == DQ_OK) fblob = (uint8_t*)p;
    if (rc == DQ_OK &&
        (rc = cache_alloc(device, sizeof(SweepJob) * std::max<size_t>(1, kf * G), &p)) == DQ_OK)
      d_jobs = (SweepJob*)p;
  }
  if (rc == DQ_OK) {
    cu(cudaMemcpyAsync(fblob, fall.p, fall_bytes, cudaMemcpyHostToDevice, st), "copy programs");
    cu(cudaMemsetAsync(ctr, 0, sizeof(unsigned) * G, st), "memset");
  }
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  for (auto& e : ev) cu(cudaEventCreate(&e), "cudaEventCreate");
  std::vector<double> host(sl * G);
  mark("setup");
  for (uint64_t g0 = 0; g0 < nsets && rc == DQ_OK; g0 += G) {
    const uint64_t g1 = std::min(nsets, g0 + G), ng = g1 - g0;
    ++acc.groups;
    // forward: sweep k of every set of the group in one launch per run width
    struct Range { size_t begin, end; uint32_t run_bits, max_bytes, flags; };
    std::vector<SweepJob> jobs;
    std::vector<Range> ranges;
    for (size_t k = 0; k < kf; ++k)
      for (uint32_t rbits : {5u, 3u}) {
        const size_t b0 = jobs.size();
        uint32_t mb = 0, fl = ~0u;
        for (uint64_t s = g0; s < g1; ++s) {
          if (k >= plans[s].foffs.size()) continue;
          const uint8_t* hp = plans[s].fblob.data() + plans[s].foffs[k];
          if (sweep_run_bits(hp) != rbits) continue;
          const uint32_t pb = sweep_prog_bytes(hp);
          mb = std::max(mb, pb);
          fl &= sweep_flags(hp);
          jobs.push_back(SweepJob{psi + (s - g0) * len, fblob + fbase[s] + plans[s].foffs[k],
                                  k == 0 ? (long long)plans[s].synth : -1LL, pb, 0});
        }
        if (jobs.size() > b0) ranges.push_back(Range{b0, jobs.size(), rbits, mb, fl});
      }
    if (!jobs.empty())
      cu(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(SweepJob) * jobs.size(), cudaMemcpyHostToDevice, st),
         "copy jobs");
    cu(cudaEventRecord(ev[0], st), "event");
    for (const Range& r : ranges) {
      if (rc != DQ_OK) break;
      rc = launch_sweep_multi(d_jobs + r.begin, (uint32_t)(r.end - r.begin), n, rb, r.run_bits,
                              r.max_bytes, st, r.flags);
      ++acc.launches;
    }
    for (uint64_t s = g0; s < g1 && rc == DQ_OK; ++s) {
      double2* ps = psi + (s - g0) * len;
      if (plans[s].foffs.empty()) {  // no sweep: the state is a basis vector
        rc = launch_set_basis(ps, n, (uint64_t)std::max<int64_t>(plans[s].synth, 0), st, device);
        ++acc.launches;
      }
      uint64_t extra = 0;
      if (rc == DQ_OK) rc = materialize_perm(ps, n, plans[s].perm, st, &extra);
      acc.launches += extra;
    }
    cu(cudaEventRecord(ev[1], st), "event");
    mark("forward enqueue");
    // lambda = H psi and E for every set of the group
    if (rc == DQ_OK) {
      k_pauli_multi<<<dim3(pblocks, (unsigned)ng), kRedThreads, 0, st>>>(
          psi, lam, len, t.groups, t.ngroups, t.terms, part, ctr, slots + nslots, sl);
      cu(cudaGetLastError(), "k_pauli_multi");
      ++acc.launches;
    }
    cu(cudaEventRecord(ev[2], st), "event");
    // backward: sweep k of every set of the group in one launch
    if (rc == DQ_OK) {
      std::vector<double2*> pp(ng), lp(ng);
      std::vector<double*> sp(ng);
      for (uint64_t s = 0; s < ng; ++s) {
        pp[s] = psi + s * len;
        lp[s] = lam + s * len;
        sp[s] = slots + s * sl;
      }
      std::vector<ABatchSet> bs;
      bs.reserve(ng);
      for (uint64_t s = g0; s < g1; ++s) bs.push_back(std::move(plans[s].back));
      uint64_t nl = 0;
      mark("observable enqueue");
      rc = adjoint_backward_batch(pp.data(), lp.data(), bs, sp.data(), st, device, &nl);
      acc.launches += nl;
      mark("backward (host)");
    }
    cu(cudaEventRecord(ev[3], st), "event");
    if (rc == DQ_OK)
      cu(cudaMemcpyAsync(host.data(), slots, sizeof(double) * sl * ng, cudaMemcpyDeviceToHost, st),
         "copy slots");
    cu(cudaStreamSynchronize(st), "sync");
    mark("sync");
    if (rc == DQ_OK) {
      float a = 0.f, b = 0.f, c = 0.f;
      cudaEventElapsedTime(&a, ev[0], ev[1]);
      cudaEventElapsedTime(&b, ev[1], ev[2]);
      cudaEventElapsedTime(&c, ev[2], ev[3]);
      acc.forward_ms += a;
      acc.observable_ms += b;
      acc.backward_ms += c;
      for (uint64_t s = g0; s < g1; ++s) {
        const double* h = host.data() + (s - g0) * sl;
        expvals[s] = h[nslots];
        double* gr = nparams ? grads + s * nparams : nullptr;
        for (uint64_t p = 0; p < nparams; ++p) gr[p] = 0.0;
        uint64_t k = 0;
        for (uint64_t i = 0; i < ninst; ++i) {
          if (!param_index || is_noop_kind(prog[i].kind)) continue;
          for (int j = 0; j < 4; ++j) {
            const int32_t v = param_index[4 * i + j];
            if (v >= 0) gr[v] += 2.0 * h[k++];
          }
        }
      }
    }
  }
  cudaStreamSynchronize(st);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  free_terms(t, st);
  cudaStreamSynchronize(st);
  if (psi) cache_free(device, sizeof(double2) * len * G, psi);
  if (lam) cache_free(device, sizeof(double2) * len * G, lam);
  if (slots) cache_free(device, sizeof(double) * sl * G, slots);
  if (part) cache_free(device, sizeof(double) * pblocks * G, part);
  if (ctr) cache_free(device, sizeof(unsigned) * G, ctr);
  if (fblob) cache_free(device, fall_bytes, fblob);
  if (d_jobs) cache_free(device, sizeof(SweepJob) * std::max<size_t>(1, kf * G), d_jobs);
  cudaStreamDestroy(st);
  mark("gradients+finish");
  acc.batched = 1;
  if (stats) *stats = acc;
  return rc;
}

}  // extern "C"
