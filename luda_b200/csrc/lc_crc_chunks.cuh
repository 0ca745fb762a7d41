// Masked CRC32C of one large buffer, split over many CTAs.
//
// Each CTA computes the raw CRC register (zero initial value, no final
// inversion) of one chunk into partials[c]; the CTA that finishes last (an
// atomic ticket, no waiting) combines the partials:
//   crc(data) = XOR_c shift(partial_c, bytes after chunk c)
//               XOR shift(0xffffffff, n) XOR 0xffffffff
// where shift(r, m) multiplies r by x^(8m) mod P in GF(2)[x] (feeding m zero
// bytes).  The result is stored as crc32c::Mask(crc) (util/crc32c.h:29-32),
// i.e. what LevelDB writes in a block trailer.  The powers x^(8*2^k) mod P are
// built per CTA by squaring, so the kernel needs no table in global memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lc {

constexpr uint32_t kCrcChunkBytes = 64 * 1024;
constexpr uint32_t kCrcChunkThreads = 256;

__device__ __forceinline__ uint32_t crcc_mulmod(uint32_t a, uint32_t b) {
  uint32_t p = 0;
  for (int i = 0; i < 32; i++) {
    if (a & 0x80000000u) p ^= b;
    a <<= 1;
    b = (b & 1) ? (b >> 1) ^ 0x82F63B78u : (b >> 1);
  }
  return p;
}

// r * x^(8m) mod P using pow2[k] = x^(8*2^k) mod P.
__device__ __forceinline__ uint32_t crcc_shift(const uint32_t* pow2, uint32_t r, uint64_t m) {
  for (int k = 0; m; k++, m >>= 1)
    if (m & 1) r = crcc_mulmod(pow2[k], r);
  return r;
}

// Body shared by every kernel that computes a chunked CRC.  `counter` must be
// zero before the launch; the last CTA leaves it at zero again.
__device__ __forceinline__ void crc32c_chunks_body(const uint8_t* data, uint64_t n,
                                                   uint32_t* partials, uint32_t* counter,
                                                   uint32_t* out) {
  __shared__ uint32_t tab[256];
  __shared__ uint32_t pow2[64];
  __shared__ uint32_t red[kCrcChunkThreads / 32];
  __shared__ bool last;
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = i;
    for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ 0x82F63B78u : (c >> 1);
    tab[i] = c;
  }
  if (threadIdx.x == 0) {
    uint32_t x8 = 0x80000000u;  // x^0
    for (int b = 0; b < 8; b++) x8 = (x8 & 1) ? (x8 >> 1) ^ 0x82F63B78u : (x8 >> 1);
    pow2[0] = x8;  // x^8
    for (int k = 1; k < 64; k++) pow2[k] = crcc_mulmod(pow2[k - 1], pow2[k - 1]);
  }
  __syncthreads();
  const uint64_t c0 = (uint64_t)blockIdx.x * kCrcChunkBytes;
  const uint64_t c1 = c0 + kCrcChunkBytes < n ? c0 + kCrcChunkBytes : n;
  const uint64_t len = c1 > c0 ? c1 - c0 : 0;
  const uint64_t seg = (len + blockDim.x - 1) / blockDim.x;
  const uint64_t b = c0 + (uint64_t)threadIdx.x * seg;
  const uint64_t e = b + seg < c1 ? b + seg : c1;
  uint32_t r = 0;
  for (uint64_t i = b; i < e; i++) r = tab[(r ^ data[i]) & 0xff] ^ (r >> 8);
  uint32_t v = b < c1 ? crcc_shift(pow2, r, c1 - e) : 0;
  for (int o = 16; o > 0; o >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t x = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; w++) x ^= red[w];
    partials[blockIdx.x] = x;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  // the last CTA combines every chunk's register
  __threadfence();
  uint32_t acc = 0;
  for (uint32_t c = threadIdx.x; c < gridDim.x; c += blockDim.x) {
    const uint64_t end = (uint64_t)(c + 1) * kCrcChunkBytes < n ? (uint64_t)(c + 1) * kCrcChunkBytes : n;
    const uint32_t p = __ldcg(partials + c);
    acc ^= crcc_shift(pow2, p, n - end);
  }
  for (int o = 16; o > 0; o >>= 1) acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t x = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; w++) x ^= red[w];
    const uint32_t full = x ^ crcc_shift(pow2, 0xffffffffu, n) ^ 0xffffffffu;
    *out = ((full >> 15) | (full << 17)) + 0xa282ead8u;
    *counter = 0;
  }
}

inline uint32_t crc32c_chunk_count(uint64_t n) {
  uint64_t c = (n + kCrcChunkBytes - 1) / kCrcChunkBytes;
  return (uint32_t)(c ? c : 1);
}

}  // namespace lc
