// dq_rng.cuh — the outcome RNG of the reference, usable on host and device.
//
// The reference draws every measurement outcome and every sampled shot from
// ChaCha8Rng::seed_from_u64(seed) (rand_chacha 0.3.1, rand_core 0.6.4) with
// rng.gen::<f64>() (rand 0.8.5), at statevector/simulator.rs:172,256,280,343
// and engine.rs:210,341,427.  Those crates are not part of the reference
// tree; their published algorithms are restated here:
//   - seed_from_u64: PCG32 XSH-RR, LCG multiplier 6364136223846793005,
//     increment 11634580027462260723, state advanced before each of the 8
//     outputs; output i is key word i (little-endian bytes of the seed).
//   - ChaCha8 block: "expand 32-byte k", key words 4..11, 64-bit block
//     counter in words 12..13, stream id 0 in words 14..15, 8 rounds, output
//     = rounds(input) + input.  Blocks are consumed in counter order.
//   - next_u64 = low word | high word << 32 from consecutive words; f64 draws
//     only ever take word pairs at even offsets, so draw s uses the words
//     2s, 2s+1 of the stream, i.e. block s/8, words 2(s%8) and 2(s%8)+1.
//   - gen::<f64>() = (next_u64 >> 11) * 2^-53.
// Because draw s depends only on (key, s), the device computes any draw
// independently; the host keeps a sequential cursor for measurement order.
#pragma once

#include <stdint.h>

namespace dq {

__host__ __device__ __forceinline__ uint32_t rotl32(uint32_t x, int k) {
  return (x << k) | (x >> (32 - k));
}

#define DQ_QR(a, b, c, d)                 \
  a += b; d ^= a; d = ::dq::rotl32(d, 16); \
  c += d; b ^= c; b = ::dq::rotl32(b, 12); \
  a += b; d ^= a; d = ::dq::rotl32(d, 8);  \
  c += d; b ^= c; b = ::dq::rotl32(b, 7);

__host__ __device__ inline void chacha_block(const uint32_t in[16], uint32_t rounds,
                                             uint32_t out[16]) {
  uint32_t x[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) x[i] = in[i];
  for (uint32_t r = 0; r < rounds; r += 2) {
    DQ_QR(x[0], x[4], x[8], x[12]);
    DQ_QR(x[1], x[5], x[9], x[13]);
    DQ_QR(x[2], x[6], x[10], x[14]);
    DQ_QR(x[3], x[7], x[11], x[15]);
    DQ_QR(x[0], x[5], x[10], x[15]);
    DQ_QR(x[1], x[6], x[11], x[12]);
    DQ_QR(x[2], x[7], x[8], x[13]);
    DQ_QR(x[3], x[4], x[9], x[14]);
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
}

__host__ __device__ inline void chacha8_stream_block(const uint32_t key[8], uint64_t counter,
                                                     uint32_t out[16]) {
  uint32_t in[16];
  in[0] = 0x61707865u;
  in[1] = 0x3320646eu;
  in[2] = 0x79622d32u;
  in[3] = 0x6b206574u;
#pragma unroll
  for (int i = 0; i < 8; ++i) in[4 + i] = key[i];
  in[12] = (uint32_t)counter;
  in[13] = (uint32_t)(counter >> 32);
  in[14] = 0;
  in[15] = 0;
  chacha_block(in, 8, out);
}

__host__ __device__ inline void seed_key_from_u64(uint64_t state, uint32_t key[8]) {
  const uint64_t mul = 6364136223846793005ULL;
  const uint64_t inc = 11634580027462260723ULL;
  for (int i = 0; i < 8; ++i) {
    state = state * mul + inc;
    const uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
    const uint32_t rot = (uint32_t)(state >> 59);
    key[i] = (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
  }
}

__host__ __device__ __forceinline__ double u64_to_f64(uint64_t v) {
  return (double)(v >> 11) * (1.0 / 9007199254740992.0);
}

// Draw number s of the stream keyed by key (independent of all other draws).
__host__ __device__ inline double chacha8_draw(const uint32_t key[8], uint64_t s) {
  uint32_t blk[16];
  chacha8_stream_block(key, s >> 3, blk);
  const int w = (int)(s & 7u) * 2;
  const uint64_t v = (uint64_t)blk[w] | ((uint64_t)blk[w + 1] << 32);
  return u64_to_f64(v);
}

// Sequential host cursor over the f64 draws (one block per 8 draws).
struct Chacha8Cursor {
  uint32_t key[8];
  uint64_t next;        // index of the next draw
  uint64_t cached_blk;  // block counter held in buf
  uint32_t buf[16];
  bool have;

  void seed(uint64_t s) {
    seed_key_from_u64(s, key);
    next = 0;
    have = false;
  }
  void set_key(const uint32_t k[8]) {
    for (int i = 0; i < 8; ++i) key[i] = k[i];
    next = 0;
    have = false;
  }
  double draw() {
    const uint64_t blk = next >> 3;
    if (!have || blk != cached_blk) {
      chacha8_stream_block(key, blk, buf);
      cached_blk = blk;
      have = true;
    }
    const int w = (int)(next & 7u) * 2;
    ++next;
    return u64_to_f64((uint64_t)buf[w] | ((uint64_t)buf[w + 1] << 32));
  }
};

}  // namespace dq
