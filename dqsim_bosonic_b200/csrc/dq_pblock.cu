// dq_pblock.cu — tensor-product merge of two block states on the device.
//
// The p-block simulator keeps one state per group of entangled qubits and
// merges two blocks when a gate spans them (merge_blocks,
// src/distributed/pblock/model.rs:35-57).  Block a holds the state of its
// ascending qubits qa[0..na), block b of qb[0..nb).  The merged block's
// qubits are the ascending union; amplitude i of the merged state is
//   a[la(i)] * b[lb(i)],
// where bit k of la(i) is the bit of i at the merged position of qa[k]
// (likewise lb for b).  The product is num-complex's (ar br - ai bi,
// ar bi + ai br) with no FMA, so the result is bit-identical to the
// reference loop.
//
// One pass: 16 B written per merged amplitude, a and b gathered (from L2 when
// the blocks are small).  The bit gathers use per-byte tables in shared
// memory: for byte c of i with value v, tab[c][v] = (la part, lb part).
#include <cuda_runtime.h>

#include <algorithm>
#include <string.h>

#include <string>
#include <vector>

#include "dq_common.cuh"
#include "dq_engine.cuh"
#include "dq_handle.cuh"

namespace dq {
namespace {

constexpr uint32_t kMergeMaxBytes = (kMaxQubits + 7) / 8;  // index bytes of a merged state

// Merged element i = a[la(i)] * b[lb(i)], the gather offsets la / lb the OR of
// one table entry per index byte.  A warp writes runs of 256 consecutive
// elements (one value of the high index bytes, looked up once per run); each
// lane keeps the low-byte entries of its 8 elements of a run (lane + 32 k) in
// registers for the whole launch, so a run costs it 8 independent gathers,
// products and stores.  States of fewer than 256 amplitudes take one thread
// per element.
__global__ void __launch_bounds__(256) k_block_merge(double2* __restrict__ out, uint64_t len,
                                                     const double2* __restrict__ a,
                                                     const double2* __restrict__ b,
                                                     const ulonglong2* __restrict__ gtab,
                                                     uint32_t nbytes) {
  __shared__ ulonglong2 tab[kMergeMaxBytes][256];
  for (uint32_t t = threadIdx.x; t < nbytes * 256u; t += blockDim.x) tab[t >> 8][t & 255u] = gtab[t];
  __syncthreads();
  if (len < 256) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
         i += (uint64_t)gridDim.x * blockDim.x) {
      const ulonglong2 e = tab[0][i];
      out[i] = cmul_x(a[e.x], b[e.y]);
    }
    return;
  }
  const uint32_t lane = threadIdx.x & 31u;
  ulonglong2 lo[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) lo[k] = tab[0][lane + 32u * k];
  const uint64_t nruns = len >> 8;
  const uint64_t wstride = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nruns; r += wstride) {
    uint64_t la = 0, lb = 0;
    for (uint32_t c = 1; c < nbytes; ++c) {
      const ulonglong2 e = tab[c][(r >> (8u * (c - 1u))) & 255u];
      la |= e.x;
      lb |= e.y;
    }
    double2* o = out + (r << 8) + lane;
    double2 x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      x[k] = a[la | lo[k].x];
      y[k] = b[lb | lo[k].y];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) o[32 * k] = cmul_x(x[k], y[k]);
  }
}

bool ascending(const uint32_t* q, uint32_t n) {
  for (uint32_t k = 1; k < n; ++k)
    if (q[k] <= q[k - 1]) return false;
  return true;
}

}  // namespace
}  // namespace dq

using namespace dq;

extern "C" {

int dq_block_merge(dq_state_t a, const uint32_t* a_qubits, uint32_t na, dq_state_t b,
                   const uint32_t* b_qubits, uint32_t nb, dq_state_t out) {
  DQ_TRY(check_handle(a));
  DQ_TRY(check_handle(b));
  DQ_TRY(check_handle_lazy(out));
  if (out == a || out == b) return fail(DQ_ERR_INVALID_ARG, "the merged block must be a third state");
  if ((na && !a_qubits) || (nb && !b_qubits)) return fail(DQ_ERR_INVALID_ARG, "null qubit list");
  if (a->n != na || b->n != nb)
    return fail(DQ_ERR_INVALID_ARG, "a block's qubit list must name one qubit per state qubit");
  if (!ascending(a_qubits, na) || !ascending(b_qubits, nb))
    return fail(DQ_ERR_INVALID_ARG, "block qubits must be ascending and distinct");
  if (a->device != out->device || b->device != out->device)
    return fail(DQ_ERR_INVALID_ARG, "blocks must live on one device");
  // merged qubits: the ascending union
  std::vector<uint32_t> u;
  u.reserve(na + nb);
  {
    uint32_t i = 0, j = 0;
    while (i < na || j < nb) {
      uint32_t q;
      if (j >= nb || (i < na && a_qubits[i] < b_qubits[j])) q = a_qubits[i++];
      else if (i >= na || b_qubits[j] < a_qubits[i]) q = b_qubits[j++];
      else { q = a_qubits[i++]; ++j; }  // a qubit in both blocks takes one merged position
      u.push_back(q);
    }
  }
  const uint32_t n = (uint32_t)u.size();
  if (out->n != n)
    return fail(DQ_ERR_INVALID_ARG, "the merged state must have one qubit per distinct block qubit (" +
                                        std::to_string(n) + ")");
  // per-byte gather tables
  const uint32_t nbytes = n ? (n + 7) / 8 : 1;
  std::vector<ulonglong2> tab((size_t)nbytes * 256);
  std::vector<int> ia(n, -1), ib(n, -1);
  for (uint32_t p = 0, i = 0, j = 0; p < n; ++p) {
    if (i < na && a_qubits[i] == u[p]) ia[p] = (int)i++;
    if (j < nb && b_qubits[j] == u[p]) ib[p] = (int)j++;
  }
  for (uint32_t c = 0; c < nbytes; ++c)
    for (uint32_t v = 0; v < 256; ++v) {
      unsigned long long la = 0, lb = 0;
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t p = 8 * c + k;
        if (p >= n || !((v >> k) & 1u)) continue;
        if (ia[p] >= 0) la |= 1ULL << ia[p];
        if (ib[p] >= 0) lb |= 1ULL << ib[p];
      }
      tab[(size_t)c * 256 + v] = make_ulonglong2(la, lb);
    }
  DeviceGuard g(out->device);
  // the blocks in their canonical layout, finished on their own streams
  {
    DeviceGuard ga(a->device);
    DQ_TRY(canonicalize(a));
    DQ_TRY(sync_stream(a));
  }
  {
    DeviceGuard gb(b->device);
    DQ_TRY(canonicalize(b));
    DQ_TRY(sync_stream(b));
  }
  out->lazy_basis = -1;
  reset_perm(out);
  // the tables go through the merged state's query buffers (pinned host and
  // device, kept by the handle): the call allocates nothing once they exist
  const size_t tab_bytes = sizeof(ulonglong2) * tab.size();
  DQ_TRY(ensure_query_buffers(out, tab_bytes, tab_bytes));
  memcpy(out->q_host, tab.data(), tab_bytes);
  ulonglong2* d_tab = reinterpret_cast<ulonglong2*>(out->q_dev);
  int rc = DQ_OK;
  cudaError_t e = cudaMemcpyAsync(d_tab, out->q_host, tab_bytes, cudaMemcpyHostToDevice, out->stream);
  if (e == cudaSuccess) {
    // persistent CTAs (as many as are resident), one warp per run of 256
    // elements at most
    static int per_sm[64];
    int& r = per_sm[out->device & 63];
    if (r == 0) {
      int v = 1;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_block_merge, 256, 0);
      r = v < 1 ? 1 : v;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, out->device);
    const uint64_t runs = out->len >> 8;
    const unsigned grid = std::min<unsigned>((unsigned)std::max<uint64_t>(1, (runs + 7) / 8),
                                             (unsigned)sms * (unsigned)r);
    k_block_merge<<<grid, 256, 0, out->stream>>>(out->amp, out->len, a->amp, b->amp, d_tab, nbytes);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) rc = fail(DQ_ERR_CUDA, std::string("block merge: ") + cudaGetErrorString(e));
  const int rs = sync_stream(out);
  return rc != DQ_OK ? rc : rs;
}

}  // extern "C"
