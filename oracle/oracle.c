/*
 * oracle.c — CPU restatement of the dqsim statevector hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py (its
 * cpu_baseline leg and the --impl reference arm) may load it, and only as the
 * checker or the baseline; the product path (dqsim_bosonic_b200) never links
 * or calls it.
 *
 * What it restates (reference paths are within the dqsim crate):
 *   src/engine.rs:24-101    apply_one_qubit (+ _seq 265-292)
 *   src/engine.rs:109-181   apply_n_qubit   (+ _seq 295-331)
 *   src/engine.rs:193-257   measure_qubit   (+ _seq 334-360)
 *   src/engine.rs:368-390   marginal_probs  (order-preserving O(2^n) scan)
 *   src/engine.rs:398-433   sample_counts
 *   src/gates.rs:18-261     gate matrices
 *   src/types.rs:148-293    gate_matrix_1q / fuse_circuit
 *   src/types.rs:348-418    Instruction::qubits (flush sets)
 *   src/monolithic/statevector/simulator.rs:386-632  run_instruction
 *   src/monolithic/statevector/simulator.rs:638-884  run_instruction_par / run_fused_par
 *   src/monolithic/statevector/simulator.rs:216-296  simulate_shots seeding
 *   src/distributed/pblock/model.rs:35-57            merge_blocks (tensor-product merge)
 * and the third-party arithmetic the path depends on (not in the reference
 * tree; versions pinned by its Cargo.lock):
 *   rand_chacha 0.3.1  ChaCha8Rng: 8-round ChaCha block function, 64-bit block
 *                      counter in words 12-13, stream id 0 in words 14-15,
 *                      output buffered as 4 blocks (64 u32 words)
 *   rand_core 0.6.4    SeedableRng::seed_from_u64 (PCG32 XSH-RR expansion of
 *                      the u64 into the 32-byte key) and BlockRng::next_u64
 *   rand 0.8.5         Standard f64: (next_u64 >> 11) * 2^-53
 *   num-complex 0.4.6  mul = (ar*br - ai*bi, ar*bi + ai*br), norm_sqr = re^2+im^2,
 *                      Complex/f64 divides each part, norm() = hypot(re, im)
 *
 * Arithmetic order follows the reference exactly (no FMA contraction: build
 * with -ffp-contract=off), so a unitary-only program reproduces the Rust
 * engine bit for bit.  The p1 sum of measure_qubit follows the sequential
 * ascending order of the n < 12 path; the reference's Rayon tree order for
 * n >= 12 is not reproducible by any implementation.
 *
 * Parity pins: the ChaCha block function is checked against RFC 8439 and an
 * independent ChaCha20 (OpenSSL via `cryptography`); the gate/engine/dispatch
 * restatement is checked against the analytic answers of the reference's own
 * tests (tests/test_distribution_e2e.py, tests/test_pblock_conditional.py).
 * No Rust toolchain exists here, so the seed_from_u64/ChaCha8 stream itself
 * is not pinned against rand_chacha output.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/dqsim_cuda.h"

typedef struct { double re, im; } cpx;

static inline cpx c_(double re, double im) { cpx z = {re, im}; return z; }
static inline cpx r_(double re) { return c_(re, 0.0); }
/* num-complex Mul for Complex<f64> */
static inline cpx cmul(cpx a, cpx b) {
  return c_(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline cpx cadd(cpx a, cpx b) { return c_(a.re + b.re, a.im + b.im); }
static inline cpx cneg(cpx a) { return c_(-a.re, -a.im); }
static inline double norm_sqr(cpx a) { return a.re * a.re + a.im * a.im; }

static int g_threads = 1;   /* 1 = sequential (parity); >1 = OpenMP baseline */

void or_set_threads(int t) {
  g_threads = t < 1 ? 1 : t;
#ifdef _OPENMP
  omp_set_num_threads(g_threads);
#endif
}
int or_get_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ======================================================================== */
/* ChaCha8Rng (rand_chacha 0.3.1) + seed_from_u64 (rand_core 0.6.4)         */
/* ======================================================================== */

static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

#define QR(a, b, c, d)                 \
  a += b; d ^= a; d = rotl32(d, 16);   \
  c += d; b ^= c; b = rotl32(b, 12);   \
  a += b; d ^= a; d = rotl32(d, 8);    \
  c += d; b ^= c; b = rotl32(b, 7);

/* ChaCha block function: out = rounds(in) + in (RFC 8439 section 2.3). */
void or_chacha_block(const uint32_t in[16], uint32_t rounds, uint32_t out[16]) {
  uint32_t x[16];
  memcpy(x, in, sizeof(x));
  for (uint32_t i = 0; i < rounds; i += 2) {
    QR(x[0], x[4], x[8], x[12]);
    QR(x[1], x[5], x[9], x[13]);
    QR(x[2], x[6], x[10], x[14]);
    QR(x[3], x[7], x[11], x[15]);
    QR(x[0], x[5], x[10], x[15]);
    QR(x[1], x[6], x[11], x[12]);
    QR(x[2], x[7], x[8], x[13]);
    QR(x[3], x[4], x[9], x[14]);
  }
  for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
}

typedef struct {
  uint32_t key[8];
  uint64_t counter;   /* next block counter to generate */
  uint32_t buf[64];   /* 4 blocks, rand_chacha's BUF_BLOCKS */
  uint32_t index;     /* next word in buf; 64 = empty */
} or_rng;

/* rand_core 0.6.4 seed_from_u64: PCG32 (XSH-RR), state advanced before each
 * output, 8 outputs written little-endian into the 32-byte seed. */
void or_seed_key(uint64_t state, uint32_t key[8]) {
  const uint64_t MUL = 6364136223846793005ULL;
  const uint64_t INC = 11634580027462260723ULL;
  for (int i = 0; i < 8; ++i) {
    state = state * MUL + INC;
    uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
    uint32_t rot = (uint32_t)(state >> 59);
    key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
  }
}

static void rng_refill(or_rng* g) {
  for (int b = 0; b < 4; ++b) {
    uint32_t in[16];
    in[0] = 0x61707865u; in[1] = 0x3320646eu; in[2] = 0x79622d32u; in[3] = 0x6b206574u;
    for (int i = 0; i < 8; ++i) in[4 + i] = g->key[i];
    uint64_t ctr = g->counter + (uint64_t)b;
    in[12] = (uint32_t)ctr; in[13] = (uint32_t)(ctr >> 32);
    in[14] = 0; in[15] = 0;
    or_chacha_block(in, 8, g->buf + 16 * b);
  }
  g->counter += 4;
  g->index = 0;
}

void or_rng_init_key(or_rng* g, const uint32_t key[8]) {
  memcpy(g->key, key, 32);
  g->counter = 0;
  g->index = 64;
}

void or_rng_init(or_rng* g, uint64_t seed) {
  uint32_t key[8];
  or_seed_key(seed, key);
  or_rng_init_key(g, key);
}

/* rand_core BlockRng::next_u64: low word first; straddles a refill when one
 * word is left. */
uint64_t or_rng_next_u64(or_rng* g) {
  if (g->index < 63) {
    uint64_t lo = g->buf[g->index], hi = g->buf[g->index + 1];
    g->index += 2;
    return (hi << 32) | lo;
  } else if (g->index >= 64) {
    rng_refill(g);
    g->index = 2;
    return ((uint64_t)g->buf[1] << 32) | g->buf[0];
  } else {
    uint64_t lo = g->buf[63];
    rng_refill(g);
    g->index = 1;
    return ((uint64_t)g->buf[0] << 32) | lo;
  }
}

uint32_t or_rng_next_u32(or_rng* g) {
  if (g->index >= 64) rng_refill(g);
  return g->buf[g->index++];
}

/* rand 0.8.5 Standard for f64: 53 high bits times 2^-53. */
double or_rng_f64(or_rng* g) {
  uint64_t v = or_rng_next_u64(g) >> 11;
  return (double)v * (1.0 / 9007199254740992.0);
}

void or_rng_f64_stream(uint64_t seed, uint64_t skip, uint64_t count, double* out) {
  or_rng g;
  or_rng_init(&g, seed);
  for (uint64_t i = 0; i < skip; ++i) (void)or_rng_next_u64(&g);
  for (uint64_t i = 0; i < count; ++i) out[i] = or_rng_f64(&g);
}

/* ======================================================================== */
/* engine.rs                                                                 */
/* ======================================================================== */

/* apply_one_qubit (engine.rs:24-101): identical arithmetic in the Rayon and
 * sequential branches; element order does not change results. */
void or_apply_one_qubit(double* st_, uint32_t n, const double* u_, uint32_t target,
                        uint64_t incl, uint64_t desired) {
  cpx* st = (cpx*)st_;
  const cpx* u = (const cpx*)u_;
  const cpx u00 = u[0], u01 = u[1], u10 = u[2], u11 = u[3];
  const uint64_t half = 1ULL << target;
  const uint64_t dim = 1ULL << n;
  const int64_t npairs = (int64_t)(dim >> 1);
#pragma omp parallel for if (g_threads > 1 && n >= 12) schedule(static)
  for (int64_t k = 0; k < npairs; ++k) {
    uint64_t i = (((uint64_t)k >> target) << (target + 1)) | ((uint64_t)k & (half - 1));
    if (incl == 0 || (i & incl) == desired) {
      uint64_t j = i | half;
      cpx a = st[i], b = st[j];
      st[i] = cadd(cmul(u00, a), cmul(u01, b));
      st[j] = cadd(cmul(u10, a), cmul(u11, b));
    }
  }
}

/* apply_n_qubit (engine.rs:109-181): dense 2^k x 2^k, qubits[0] = MSB, the
 * row sums start from 0 and add u[row][col]*v[col] for col ascending.  The
 * base indices are those with (i & mask) == 0, scanned like the reference. */
void or_apply_n_qubit(double* st_, uint32_t n, const double* u_, const uint32_t* qubits,
                      uint32_t k) {
  cpx* st = (cpx*)st_;
  const cpx* u = (const cpx*)u_;
  const uint32_t dim = 1u << k;
  const int64_t n_states = (int64_t)1 << n;
  uint64_t mask = 0;
  for (uint32_t b = 0; b < k; ++b) mask |= 1ULL << qubits[b];
  uint64_t offsets[32];
  for (uint32_t j = 0; j < dim; ++j) {
    uint64_t off = 0;
    for (uint32_t bit = 0; bit < k; ++bit)
      if ((j >> (k - 1 - bit)) & 1u) off |= 1ULL << qubits[bit];
    offsets[j] = off;
  }
#pragma omp parallel for if (g_threads > 1 && n >= 12) schedule(static)
  for (int64_t i = 0; i < n_states; ++i) {
    if (((uint64_t)i & mask) != 0) continue;
    cpx v[32], w[32];
    for (uint32_t j = 0; j < dim; ++j) v[j] = st[(uint64_t)i + offsets[j]];
    for (uint32_t row = 0; row < dim; ++row) {
      cpx acc = c_(0.0, 0.0);
      for (uint32_t col = 0; col < dim; ++col) acc = cadd(acc, cmul(u[row * dim + col], v[col]));
      w[row] = acc;
    }
    for (uint32_t j = 0; j < dim; ++j) st[(uint64_t)i + offsets[j]] = w[j];
  }
}

/* p1 of measure_qubit: sequential ascending sum (engine.rs:204-207, 337-340);
 * with threads > 1 an OpenMP reduction stands in for the Rayon tree. */
double or_p1(const double* st_, uint32_t n, uint32_t q) {
  const cpx* st = (const cpx*)st_;
  const int64_t n_states = (int64_t)1 << n;
  const uint64_t bit = 1ULL << q;
  double p1 = 0.0;
  if (g_threads > 1 && n >= 12) {
#pragma omp parallel for reduction(+ : p1) schedule(static)
    for (int64_t i = 0; i < n_states; ++i)
      if ((uint64_t)i & bit) p1 += norm_sqr(st[i]);
  } else {
    for (int64_t i = 0; i < n_states; ++i)
      if ((uint64_t)i & bit) p1 += norm_sqr(st[i]);
  }
  return p1;
}

/* collapse half of measure_qubit (engine.rs:210-256). */
void or_collapse(double* st_, uint32_t n, uint32_t q, int outcome, double p1) {
  cpx* st = (cpx*)st_;
  const int64_t n_states = (int64_t)1 << n;
  const uint64_t bit = 1ULL << q;
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
#pragma omp parallel for if (g_threads > 1 && n >= 12) schedule(static)
  for (int64_t i = 0; i < n_states; ++i) {
    int set = ((uint64_t)i & bit) != 0;
    if (set != (outcome == 1)) {
      st[i] = c_(0.0, 0.0);
    } else {
      st[i].re = st[i].re / norm;
      st[i].im = st[i].im / norm;
    }
  }
}

int or_measure(double* st, uint32_t n, uint32_t q, double r, double* p1_out) {
  double p1 = or_p1(st, n, q);
  int outcome = (r < p1) ? 1 : 0;
  or_collapse(st, n, q, outcome, p1);
  if (p1_out) *p1_out = p1;
  return outcome;
}

/* marginal_probs (engine.rs:368-390).  The reference sums, for each j, the
 * norm_sqr of matching i in ascending i; one ascending scan that adds into
 * bucket j(i) performs exactly the same additions in the same order. */
void or_marginal_probs(const double* st_, uint32_t n, const uint32_t* qubits, uint32_t k,
                       double* out) {
  const cpx* st = (const cpx*)st_;
  const uint64_t dim = 1ULL << k;
  for (uint64_t j = 0; j < dim; ++j) out[j] = 0.0;
  const uint64_t n_states = 1ULL << n;
  for (uint64_t i = 0; i < n_states; ++i) {
    uint64_t j = 0;
    for (uint32_t b = 0; b < k; ++b) j |= ((i >> qubits[b]) & 1ULL) << (k - 1 - b);
    out[j] += norm_sqr(st[i]);
  }
}

/* sample_counts (engine.rs:398-433) given the marginal probabilities:
 * sequential CDF, last entry forced to 1.0, partition_point(c < r) clamped. */
void or_sample_from_probs(const double* probs, uint32_t k, or_rng* g, uint64_t shots,
                          uint32_t* out_idx) {
  const uint64_t dim = 1ULL << k;
  double* cdf = (double*)malloc(sizeof(double) * dim);
  double acc = 0.0;
  for (uint64_t i = 0; i < dim; ++i) { acc += probs[i]; cdf[i] = acc; }
  cdf[dim - 1] = 1.0;
  for (uint64_t s = 0; s < shots; ++s) {
    double r = or_rng_f64(g);
    uint64_t lo = 0, hi = dim;   /* first index with !(cdf < r) */
    while (lo < hi) {
      uint64_t mid = lo + ((hi - lo) >> 1);
      if (cdf[mid] < r) lo = mid + 1; else hi = mid;
    }
    if (lo > dim - 1) lo = dim - 1;
    out_idx[s] = (uint32_t)lo;
  }
  free(cdf);
}

void or_sample(const double* st, uint32_t n, const uint32_t* qubits, uint32_t k,
               uint64_t seed, uint64_t shots, uint32_t* out_idx) {
  double* probs = (double*)malloc(sizeof(double) * (1ULL << k));
  or_marginal_probs(st, n, qubits, k, probs);
  or_rng g;
  or_rng_init(&g, seed);
  or_sample_from_probs(probs, k, &g, shots, out_idx);
  free(probs);
}

/* ======================================================================== */
/* gates.rs                                                                  */
/* ======================================================================== */

static void set_id(cpx* m, uint32_t dim) {
  for (uint32_t i = 0; i < dim * dim; ++i) m[i] = r_(0.0);
  for (uint32_t i = 0; i < dim; ++i) m[i * dim + i] = r_(1.0);
}

/* u3 (gates.rs:59-65) */
static void g_u3(double theta, double phi, double lam, cpx m[4]) {
  double ct = cos(theta / 2.0), st = sin(theta / 2.0);
  m[0] = r_(ct);
  m[1] = cneg(cmul(c_(cos(lam), sin(lam)), r_(st)));
  m[2] = cmul(c_(cos(phi), sin(phi)), r_(st));
  m[3] = cmul(c_(cos(phi + lam), sin(phi + lam)), r_(ct));
}

static void g_controlled(const cpx u[4], cpx m[16]) {  /* gates.rs:121-129 */
  set_id(m, 4);
  m[2 * 4 + 2] = u[0]; m[2 * 4 + 3] = u[1];
  m[3 * 4 + 2] = u[2]; m[3 * 4 + 3] = u[3];
}

/* 2x2 matrix of a fixed/parametric single-qubit kind (gates.rs:18-84).
 * Returns 0 if the kind is not a single-qubit gate. */
int or_matrix_1q(int kind, const double* p, double* out) {
  cpx* m = (cpx*)out;
  const double s = M_SQRT1_2;  /* FRAC_1_SQRT_2 */
  switch (kind) {
    case DQ_ID: case DQ_U0: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = r_(1); return 1;
    case DQ_X: m[0] = r_(0); m[1] = r_(1); m[2] = r_(1); m[3] = r_(0); return 1;
    case DQ_Y: m[0] = r_(0); m[1] = c_(0, -1); m[2] = c_(0, 1); m[3] = r_(0); return 1;
    case DQ_Z: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = r_(-1); return 1;
    case DQ_H: m[0] = r_(s); m[1] = r_(s); m[2] = r_(s); m[3] = r_(-s); return 1;
    case DQ_S: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = c_(0, 1); return 1;
    case DQ_SDG: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = c_(0, -1); return 1;
    case DQ_T: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = c_(s, s); return 1;
    case DQ_TDG: m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = c_(s, -s); return 1;
    case DQ_SX: m[0] = c_(0.5, 0.5); m[1] = c_(0.5, -0.5); m[2] = c_(0.5, -0.5); m[3] = c_(0.5, 0.5); return 1;
    case DQ_SXDG: m[0] = c_(0.5, -0.5); m[1] = c_(0.5, 0.5); m[2] = c_(0.5, 0.5); m[3] = c_(0.5, -0.5); return 1;
    case DQ_U3: case DQ_U: g_u3(p[0], p[1], p[2], m); return 1;
    case DQ_U2: g_u3(M_PI / 2.0, p[0], p[1], m); return 1;
    case DQ_U1: case DQ_P:
      m[0] = r_(1); m[1] = r_(0); m[2] = r_(0); m[3] = c_(cos(p[0]), sin(p[0])); return 1;
    case DQ_RX: {
      double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      m[0] = r_(c2); m[1] = c_(0, -s2); m[2] = c_(0, -s2); m[3] = r_(c2); return 1;
    }
    case DQ_RY: {
      double c2 = cos(p[0] / 2.0), s2 = sin(p[0] / 2.0);
      m[0] = r_(c2); m[1] = r_(-s2); m[2] = r_(s2); m[3] = r_(c2); return 1;
    }
    case DQ_RZ: {
      double phi = p[0];
      m[0] = c_(cos(-phi / 2.0), sin(-phi / 2.0)); m[1] = r_(0);
      m[2] = r_(0); m[3] = c_(cos(phi / 2.0), sin(phi / 2.0)); return 1;
    }
    default: return 0;
  }
}

/* Dense matrix and qubit list of a multi-qubit kind, exactly what
 * run_instruction hands to apply_n_qubit (simulator.rs:465-590).
 * Returns k (2..5) or 0 if the kind is not such a gate. */
int or_matrix_nq(const dq_inst* in, double* out, uint32_t* qubits) {
  cpx* m = (cpx*)out;
  const double s = M_SQRT1_2;
  cpx u[4];
  for (int i = 0; i < in->nq && i < 5; ++i) qubits[i] = (uint32_t)in->q[i];
  switch (in->kind) {
    case DQ_CX: case DQ_G_CX:
      set_id(m, 4); m[10] = r_(0); m[15] = r_(0); m[11] = r_(1); m[14] = r_(1); return 2;
    case DQ_CZ: case DQ_G_CZ: set_id(m, 4); m[15] = r_(-1); return 2;
    case DQ_CY:
      set_id(m, 4); m[10] = r_(0); m[15] = r_(0); m[11] = c_(0, -1); m[14] = c_(0, 1); return 2;
    case DQ_CH:
      set_id(m, 4); m[10] = r_(s); m[11] = r_(s); m[14] = r_(s); m[15] = r_(-s); return 2;
    case DQ_SWAP:
      set_id(m, 4); m[5] = r_(0); m[10] = r_(0); m[6] = r_(1); m[9] = r_(1); return 2;
    case DQ_CSX:
      set_id(m, 4);
      m[10] = c_(0.5, 0.5); m[11] = c_(0.5, -0.5); m[14] = c_(0.5, -0.5); m[15] = c_(0.5, 0.5);
      return 2;
    case DQ_CRX: { double pp[1] = {in->p[0]}; or_matrix_1q(DQ_RX, pp, (double*)u); g_controlled(u, m); return 2; }
    case DQ_CRY: { double pp[1] = {in->p[0]}; or_matrix_1q(DQ_RY, pp, (double*)u); g_controlled(u, m); return 2; }
    case DQ_CRZ: { double pp[1] = {in->p[0]}; or_matrix_1q(DQ_RZ, pp, (double*)u); g_controlled(u, m); return 2; }
    case DQ_CU1: case DQ_CP: {
      double pp[1] = {in->p[0]}; or_matrix_1q(DQ_U1, pp, (double*)u); g_controlled(u, m); return 2;
    }
    case DQ_CU3: g_u3(in->p[0], in->p[1], in->p[2], u); g_controlled(u, m); return 2;
    case DQ_CU: {  /* gates.rs:137-143 */
      cpx inner[4], phase = c_(cos(in->p[3]), sin(in->p[3]));
      g_u3(in->p[0], in->p[1], in->p[2], inner);
      for (int i = 0; i < 4; ++i) u[i] = cmul(phase, inner[i]);
      g_controlled(u, m);
      return 2;
    }
    case DQ_RXX: {  /* gates.rs:145-154 */
      double cv = cos(in->p[0] / 2.0), sv = sin(in->p[0] / 2.0);
      for (int i = 0; i < 16; ++i) m[i] = r_(0);
      m[0] = r_(cv); m[3] = c_(0, -sv);
      m[5] = r_(cv); m[6] = c_(0, -sv);
      m[9] = c_(0, -sv); m[10] = r_(cv);
      m[12] = c_(0, -sv); m[15] = r_(cv);
      return 2;
    }
    case DQ_RZZ: {  /* gates.rs:155-160 */
      double h = in->p[0] / 2.0;
      cpx ep = c_(cos(h), sin(h)), em = c_(cos(h), -sin(h));
      for (int i = 0; i < 16; ++i) m[i] = r_(0);
      m[0] = em; m[5] = ep; m[10] = ep; m[15] = em;
      return 2;
    }
    case DQ_G_PSI_MINUS: case DQ_G_PSI_PLUS: {  /* gates.rs:224-246 */
      const double pm[16] = {0, s, 0, s, s, 0, s, 0, -s, 0, s, 0, 0, -s, 0, s};
      for (int i = 0; i < 16; ++i) m[i] = r_(pm[i]);
      if (in->kind == DQ_G_PSI_PLUS)
        for (int i = 8; i < 16; ++i) m[i] = cneg(m[i]);
      return 2;
    }
    case DQ_G_PHI_PLUS: {  /* gates.rs:248-258 */
      const double pp[16] = {s, 0, s, 0, 0, s, 0, s, 0, s, 0, -s, s, 0, -s, 0};
      for (int i = 0; i < 16; ++i) m[i] = r_(pp[i]);
      return 2;
    }
    case DQ_CCX:
      set_id(m, 8); m[6 * 8 + 6] = r_(0); m[7 * 8 + 7] = r_(0); m[6 * 8 + 7] = r_(1); m[7 * 8 + 6] = r_(1);
      return 3;
    case DQ_CSWAP:
      set_id(m, 8); m[5 * 8 + 5] = r_(0); m[6 * 8 + 6] = r_(0); m[5 * 8 + 6] = r_(1); m[6 * 8 + 5] = r_(1);
      return 3;
    case DQ_RCCX:
      set_id(m, 8); m[6 * 8 + 6] = r_(0); m[7 * 8 + 7] = r_(0); m[6 * 8 + 7] = c_(0, 1); m[7 * 8 + 6] = c_(0, -1);
      return 3;
    case DQ_RC3X:
      set_id(m, 16); m[14 * 16 + 14] = c_(0, 1); m[14 * 16 + 15] = r_(0); m[15 * 16 + 14] = r_(0);
      m[15 * 16 + 15] = c_(0, -1);
      return 4;
    case DQ_C3X:
      set_id(m, 16); m[14 * 16 + 14] = r_(0); m[15 * 16 + 15] = r_(0); m[14 * 16 + 15] = r_(1);
      m[15 * 16 + 14] = r_(1);
      return 4;
    case DQ_C3SQRTX:
      set_id(m, 16);
      m[14 * 16 + 14] = c_(0.5, 0.5); m[14 * 16 + 15] = c_(0.5, -0.5);
      m[15 * 16 + 14] = c_(0.5, -0.5); m[15 * 16 + 15] = c_(0.5, 0.5);
      return 4;
    case DQ_C4X:
      set_id(m, 32); m[30 * 32 + 30] = r_(0); m[31 * 32 + 31] = r_(0); m[30 * 32 + 31] = r_(1);
      m[31 * 32 + 30] = r_(1);
      return 5;
    default:
      return 0;
  }
}

/* ======================================================================== */
/* dispatcher                                                                */
/* ======================================================================== */

typedef struct {
  double* st;
  uint32_t n;
  int32_t* cbits;
  uint64_t ncbits;
  or_rng rng;
  int sem;
  int64_t failed;
} or_ctx;

static int cond_ok(const or_ctx* c, const dq_inst* in, const dq_cond* conds) {
  for (uint32_t ci = 0; ci < in->cond_count; ++ci) {
    const dq_cond* cd = &conds[in->cond_first + ci];
    uint64_t actual = 0;
    for (uint64_t b = 0; b < cd->creg_size; ++b) {
      uint64_t idx = cd->creg_base + b;
      uint64_t val = (idx < c->ncbits && c->cbits[idx] > 0) ? (uint64_t)c->cbits[idx] : 0;
      actual |= val << b;
    }
    if (actual != cd->creg_value) return 0;
  }
  return 1;
}

static int do_measure(or_ctx* c, uint32_t q) {
  double r = or_rng_f64(&c->rng);
  return or_measure(c->st, c->n, q, r, NULL);
}

/* One instruction (conditions already checked).  Returns DQ_OK or an error. */
static int exec_inst(or_ctx* c, const dq_inst* in) {
  double mbuf[32 * 32 * 2];
  uint32_t qs[5];
  switch (in->kind) {
    case DQ_ID: case DQ_U0: case DQ_BARRIER: case DQ_CLASSICAL: case DQ_G_NOOP:
      return DQ_OK;
    case DQ_G_OPAQUE:
      return c->sem == DQ_SEM_SHOTS ? DQ_OK : DQ_ERR_UNSUPPORTED;
    case DQ_G_UNSUPPORTED:
      return DQ_ERR_UNSUPPORTED;
    case DQ_MEASURE: {
      int o = do_measure(c, (uint32_t)in->q[0]);
      if ((uint64_t)in->cbit < c->ncbits) c->cbits[in->cbit] = o;
      return DQ_OK;
    }
    case DQ_RESET: {
      int o = do_measure(c, (uint32_t)in->q[0]);
      if (o == 1) {
        or_matrix_1q(DQ_X, NULL, mbuf);
        or_apply_one_qubit(c->st, c->n, mbuf, (uint32_t)in->q[0], 0, 0);
      }
      return DQ_OK;
    }
    default:
      break;
  }
  if (or_matrix_1q(in->kind, in->p, mbuf)) {
    or_apply_one_qubit(c->st, c->n, mbuf, (uint32_t)in->q[0], 0, 0);
    return DQ_OK;
  }
  int k = or_matrix_nq(in, mbuf, qs);
  if (k == 0) return DQ_ERR_INTERNAL;
  or_apply_n_qubit(c->st, c->n, mbuf, qs, (uint32_t)k);
  return DQ_OK;
}

/* StatevectorSimulator::simulate instruction loop (simulator.rs:337-356):
 * the caller provides st = |0...0> (or any start state) of 2^n amplitudes. */
int or_run(double* st, uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
           uint64_t seed, int32_t* cbits, uint64_t ncbits, int64_t* failed) {
  or_ctx c;
  c.st = st; c.n = n; c.cbits = cbits; c.ncbits = ncbits; c.sem = DQ_SEM_SIMULATE;
  or_rng_init(&c.rng, seed);
  for (uint64_t i = 0; i < ninst; ++i) {
    if (!cond_ok(&c, &prog[i], conds)) continue;
    int rc = exec_inst(&c, &prog[i]);
    if (rc != DQ_OK) { if (failed) *failed = (int64_t)i; return rc; }
  }
  if (failed) *failed = -1;
  return DQ_OK;
}

/* ---- fuse_circuit (types.rs:239-293) ------------------------------------ */

/* A fused program entry: either an original instruction index or a fused 2x2. */
typedef struct {
  int64_t inst;     /* >= 0: original instruction; -1: fused matrix */
  uint32_t qubit;
  cpx m[4];
} or_fused;

static void matmul2(const cpx a[4], const cpx b[4], cpx out[4]) {  /* types.rs:148-160 */
  cpx r0 = cadd(cmul(a[0], b[0]), cmul(a[1], b[2]));
  cpx r1 = cadd(cmul(a[0], b[1]), cmul(a[1], b[3]));
  cpx r2 = cadd(cmul(a[2], b[0]), cmul(a[3], b[2]));
  cpx r3 = cadd(cmul(a[2], b[1]), cmul(a[3], b[3]));
  out[0] = r0; out[1] = r1; out[2] = r2; out[3] = r3;
}

static int is_identity2(const cpx m[4]) {  /* types.rs:239-244 */
  return hypot(m[0].re - 1.0, m[0].im) < 1e-10 && hypot(m[1].re, m[1].im) < 1e-10 &&
         hypot(m[2].re, m[2].im) < 1e-10 && hypot(m[3].re - 1.0, m[3].im) < 1e-10;
}

/* Instruction::qubits (types.rs:348-418) of an unconditional or conditional
 * instruction (a conditional touches its op's qubits). */
static int inst_touched(const dq_inst* in, uint32_t* out) {
  switch (in->kind) {
    case DQ_BARRIER: case DQ_CLASSICAL: return 0;
    default: break;
  }
  int nq = in->nq;
  if (nq > DQ_MAX_INST_QUBITS) nq = DQ_MAX_INST_QUBITS;
  for (int i = 0; i < nq; ++i) out[i] = (uint32_t)in->q[i];
  return nq;
}

/* Returns the number of fused entries written to out (capacity ninst + n).
 * Fusable: unconditional single-qubit gates (gate_matrix_1q, types.rs:164-237).
 * The final flush visits pending qubits in ascending order (the reference
 * iterates a HashMap; the final flush only affects the discarded end state). */
uint64_t or_fuse(const dq_inst* prog, uint64_t ninst, uint32_t n, or_fused* out) {
  cpx* pend = (cpx*)malloc(sizeof(cpx) * 4 * (n ? n : 1));
  char* has = (char*)calloc(n ? n : 1, 1);
  uint64_t no = 0;
  for (uint64_t i = 0; i < ninst; ++i) {
    const dq_inst* in = &prog[i];
    cpx m[4];
    if (in->cond_count == 0 && or_matrix_1q(in->kind, in->p, (double*)m)) {
      uint32_t q = (uint32_t)in->q[0];
      if (!has[q]) {
        has[q] = 1;
        pend[4 * q + 0] = r_(1); pend[4 * q + 1] = r_(0);
        pend[4 * q + 2] = r_(0); pend[4 * q + 3] = r_(1);
      }
      matmul2(m, &pend[4 * q], &pend[4 * q]);
    } else {
      uint32_t touched[DQ_MAX_INST_QUBITS];
      int nt = inst_touched(in, touched);
      for (int t = 0; t < nt; ++t) {
        uint32_t q = touched[t];
        if (q < n && has[q]) {
          has[q] = 0;
          if (!is_identity2(&pend[4 * q])) {
            out[no].inst = -1; out[no].qubit = q;
            memcpy(out[no].m, &pend[4 * q], sizeof(cpx) * 4);
            ++no;
          }
        }
      }
      out[no].inst = (int64_t)i; out[no].qubit = 0;
      ++no;
    }
  }
  for (uint32_t q = 0; q < n; ++q) {
    if (has[q] && !is_identity2(&pend[4 * q])) {
      out[no].inst = -1; out[no].qubit = q;
      memcpy(out[no].m, &pend[4 * q], sizeof(cpx) * 4);
      ++no;
    }
  }
  free(pend);
  free(has);
  return no;
}

/* Fused program as flat arrays for tests: inst index (-1 = fused), qubit, 2x2. */
uint64_t or_fuse_export(const dq_inst* prog, uint64_t ninst, uint32_t n, int64_t* inst_out,
                        uint32_t* qubit_out, double* mat_out) {
  or_fused* f = (or_fused*)malloc(sizeof(or_fused) * (ninst + n + 1));
  uint64_t nf = or_fuse(prog, ninst, n, f);
  for (uint64_t i = 0; i < nf; ++i) {
    inst_out[i] = f[i].inst;
    qubit_out[i] = f[i].qubit;
    memcpy(mat_out + 8 * i, f[i].m, sizeof(cpx) * 4);
  }
  free(f);
  return nf;
}

/* One shot of simulate_shots (simulator.rs:277-285): fused program, shots
 * semantics, rng = seed_from_u64(base_seed.wrapping_add(i)). */
static int run_one_shot(const or_fused* f, uint64_t nf, const dq_inst* prog, const dq_cond* conds,
                        uint32_t n, uint64_t seed, double* st, int32_t* cbits, uint64_t ncbits,
                        int64_t* failed) {
  const uint64_t dim = 1ULL << n;
  memset(st, 0, sizeof(double) * 2 * dim);
  st[0] = 1.0;
  for (uint64_t i = 0; i < ncbits; ++i) cbits[i] = -1;
  or_ctx c;
  c.st = st; c.n = n; c.cbits = cbits; c.ncbits = ncbits; c.sem = DQ_SEM_SHOTS;
  or_rng_init(&c.rng, seed);
  for (uint64_t e = 0; e < nf; ++e) {
    if (f[e].inst < 0) {
      or_apply_one_qubit(st, n, (const double*)f[e].m, f[e].qubit, 0, 0);
      continue;
    }
    const dq_inst* in = &prog[f[e].inst];
    if (!cond_ok(&c, in, conds)) continue;
    int rc = exec_inst(&c, in);
    if (rc != DQ_OK) { if (failed) *failed = f[e].inst; return rc; }
  }
  return DQ_OK;
}

/* simulate_shots: writes per-shot classical registers (0/1, -1 = unwritten)
 * into cbits_out[shot * ncbits + b].  Shots run in parallel when threads > 1
 * (each shot sequential, like the reference's per-shot _seq kernels). */
int or_run_shots(uint32_t n, const dq_inst* prog, uint64_t ninst, const dq_cond* conds,
                 uint64_t base_seed, uint64_t shot0, uint64_t shots, int32_t* cbits_out,
                 uint64_t ncbits, int64_t* failed) {
  or_fused* f = (or_fused*)malloc(sizeof(or_fused) * (ninst + n + 1));
  uint64_t nf = or_fuse(prog, ninst, n, f);
  const int saved = g_threads;
  int rc_all = DQ_OK;
  int64_t fail_all = -1;
  const int par = saved > 1;
  g_threads = 1;  /* sequential kernels inside each shot */
#pragma omp parallel for if (par) schedule(dynamic, 1)
  for (int64_t s = 0; s < (int64_t)shots; ++s) {
    double* st = (double*)malloc(sizeof(double) * 2 * (1ULL << n));
    int64_t fl = -1;
    int rc = run_one_shot(f, nf, prog, conds, n, base_seed + shot0 + (uint64_t)s, st,
                          cbits_out + (uint64_t)s * ncbits, ncbits, &fl);
    if (rc != DQ_OK) {
#pragma omp critical
      { rc_all = rc; fail_all = fl; }
    }
    free(st);
  }
  g_threads = saved;
  free(f);
  if (failed) *failed = fail_all;
  return rc_all;
}

/* <psi|H|psi> for H = sum_t coeff_t * P_t (dq_pauli_term convention of
 * include/dqsim_cuda.h: P = i^{ny} X^x Z^z, Y on qubits with both bits).
 * No reference counterpart (the reference has no observables); used as the
 * checker of the engine's observables and, through or_run, of its adjoint
 * gradients (parameter shift and finite differences on the CPU).  Plain
 * ascending loops; terms are summed in the order given. */
double or_expval_pauli(const double* st_, uint32_t n, const dq_pauli_term* terms,
                       uint64_t nterms) {
  const cpx* st = (const cpx*)st_;
  const uint64_t len = 1ULL << n;
  double total = 0.0;
  for (uint64_t t = 0; t < nterms; ++t) {
    const uint64_t x = terms[t].xmask, z = terms[t].zmask;
    const int ny = __builtin_popcountll(x & z) & 3;
    double re = 0.0, im = 0.0; /* sum_j conj(psi_j) (X^x Z^z psi)_j */
    for (uint64_t j = 0; j < len; ++j) {
      const uint64_t src = j ^ x;
      const double sgn = (__builtin_popcountll(src & z) & 1) ? -1.0 : 1.0;
      const cpx a = st[j], b = st[src];
      re += sgn * (a.re * b.re + a.im * b.im);
      im += sgn * (a.re * b.im - a.im * b.re);
    }
    /* multiply by i^ny and keep the real part */
    double v;
    switch (ny) {
      case 0: v = re; break;
      case 1: v = -im; break;
      case 2: v = -re; break;
      default: v = im; break;
    }
    total += terms[t].coeff * v;
  }
  return total;
}

/* merge_blocks (src/distributed/pblock/model.rs:35-57): merged qubits = the
 * ascending union of qa[0..na) and qb[0..nb) (both ascending); for every
 * merged index i, a_local gathers the bits of i at the merged positions of
 * a's qubits, likewise b_local; out[i] = a[a_local] * b[b_local] (num-complex
 * multiplication).  out has 2^|union| entries; returns |union|. */
uint32_t or_block_merge(const double* a_, const uint32_t* qa, uint32_t na, const double* b_,
                        const uint32_t* qb, uint32_t nb, double* out_) {
  uint32_t u[128];
  uint32_t n = 0, i = 0, j = 0;
  while (i < na || j < nb) {
    if (j >= nb || (i < na && qa[i] < qb[j])) u[n++] = qa[i++];
    else if (i >= na || qb[j] < qa[i]) u[n++] = qb[j++];
    else { u[n++] = qa[i++]; ++j; }
  }
  const cpx* a = (const cpx*)a_;
  const cpx* b = (const cpx*)b_;
  cpx* out = (cpx*)out_;
  uint32_t pa[64], pb[64];
  for (uint32_t k = 0; k < na; ++k)
    for (uint32_t p = 0; p < n; ++p)
      if (u[p] == qa[k]) pa[k] = p;
  for (uint32_t k = 0; k < nb; ++k)
    for (uint32_t p = 0; p < n; ++p)
      if (u[p] == qb[k]) pb[k] = p;
  const uint64_t dim = 1ULL << n;
  for (uint64_t x = 0; x < dim; ++x) {
    uint64_t la = 0, lb = 0;
    for (uint32_t k = 0; k < na; ++k)
      if ((x >> pa[k]) & 1ULL) la |= 1ULL << k;
    for (uint32_t k = 0; k < nb; ++k)
      if ((x >> pb[k]) & 1ULL) lb |= 1ULL << k;
    out[x] = cmul(a[la], b[lb]);
  }
  return n;
}
