// Device-side codecs and comparisons for the LevelDB table format.
//
// Restated from the reference's host code: varint/fixed codecs
// (util/coding.cc:9-192), the internal-key order (db/dbformat.cc:51-67), the
// bloom hash (util/hash.cc:22-51) and CRC32C (util/crc32c.cc:276; reflected
// Castagnoli polynomial 0x82F63B78 with pre/post inversion).  The CRC is
// computed from tables built from the polynomial (a 256-entry byte table, or
// the field tables of the row CRC) and combined across lanes with
// multiplication by x^(8n) mod P in GF(2)[x].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lc_job.h"

namespace lc {

constexpr uint32_t kCrcPoly = 0x82F63B78u;
constexpr uint64_t kSeekTag = (((1ull << 56) - 1) << 8) | 1ull;  // PackSequenceAndType(kMax, kTypeValue)
constexpr uint32_t kFilterBaseLg = 11;                             // table/filter_block.cc:14
constexpr uint32_t kTrailer = 5;                                   // type byte + crc
constexpr uint32_t kFooter = 48;                                   // table/format.h:61

__device__ __forceinline__ uint32_t ld_le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
__device__ __forceinline__ uint64_t ld_le64(const uint8_t* p) {
  return (uint64_t)ld_le32(p) | ((uint64_t)ld_le32(p + 4) << 32);
}
__device__ __forceinline__ void st_le32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v;
  p[1] = (uint8_t)(v >> 8);
  p[2] = (uint8_t)(v >> 16);
  p[3] = (uint8_t)(v >> 24);
}

// LEB128 decode bounded by `lim`; nullptr on truncation or overlong input.
__device__ __forceinline__ const uint8_t* get_varint32(const uint8_t* p, const uint8_t* lim,
                                                       uint32_t* v) {
  uint32_t r = 0;
  for (uint32_t shift = 0; shift <= 28 && p < lim; shift += 7) {
    uint32_t b = *p++;
    if (b & 128) {
      r |= (b & 127) << shift;
    } else {
      *v = r | (b << shift);
      return p;
    }
  }
  return nullptr;
}
__device__ __forceinline__ const uint8_t* get_varint64(const uint8_t* p, const uint8_t* lim,
                                                       uint64_t* v) {
  uint64_t r = 0;
  for (uint32_t shift = 0; shift <= 63 && p < lim; shift += 7) {
    uint64_t b = *p++;
    if (b & 128) {
      r |= (b & 127) << shift;
    } else {
      *v = r | (b << shift);
      return p;
    }
  }
  return nullptr;
}
__host__ __device__ __forceinline__ uint32_t varint_len(uint64_t v) {
  uint32_t n = 1;
  while (v >= 128) {
    v >>= 7;
    n++;
  }
  return n;
}
// 32-bit forms of the two above (no 64-bit shifts or compares).
__device__ __forceinline__ uint32_t varint_len32(uint32_t v) {
  return 1u + (v >= (1u << 7)) + (v >= (1u << 14)) + (v >= (1u << 21)) + (v >= (1u << 28));
}
__device__ __forceinline__ uint8_t* put_varint32(uint8_t* p, uint32_t v) {
  while (v >= 128) {
    *p++ = (uint8_t)(v | 128);
    v >>= 7;
  }
  *p++ = (uint8_t)v;
  return p;
}
__device__ __forceinline__ uint8_t* put_varint(uint8_t* p, uint64_t v) {
  while (v >= 128) {
    *p++ = (uint8_t)(v | 128);
    v >>= 7;
  }
  *p++ = (uint8_t)v;
  return p;
}

// Bytewise comparison (Slice::compare): memcmp, then length.
__device__ __forceinline__ int bytes_cmp(const uint8_t* a, uint32_t al, const uint8_t* b,
                                         uint32_t bl) {
  uint32_t m = al < bl ? al : bl;
  for (uint32_t i = 0; i < m; i++) {
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  }
  return al < bl ? -1 : (al > bl ? 1 : 0);
}

// InternalKeyComparator::Compare (db/dbformat.cc:51-67).
__device__ __forceinline__ int ikey_cmp(const uint8_t* a, uint32_t al, const uint8_t* b,
                                        uint32_t bl) {
  int r = bytes_cmp(a, al - 8, b, bl - 8);
  if (r == 0) {
    uint64_t an = ld_le64(a + al - 8), bn = ld_le64(b + bl - 8);
    r = an > bn ? -1 : (an < bn ? 1 : 0);
  }
  return r;
}

// Big-endian value of the first 8 user-key bytes, zero padded: equal prefixes
// say nothing, different prefixes order the keys.
__device__ __forceinline__ uint64_t user_prefix(const uint8_t* k, uint32_t klen) {
  uint32_t u = klen - 8;
  uint64_t v = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) v = (v << 8) | (uint64_t)((uint32_t)i < u ? k[i] : 0);
  return v;
}

// The 8 user-key bytes after the first `skip`, big endian, zero padded: the
// prefix of an entry when every key of the job shares its first `skip` bytes.
__device__ __forceinline__ uint64_t user_prefix_after(const uint8_t* k, uint32_t klen,
                                                      uint32_t skip) {
  const uint32_t u = klen - 8;
  uint64_t v = 0;
#pragma unroll
  for (uint32_t i = 0; i < 8; i++) v = (v << 8) | (uint64_t)(skip + i < u ? k[skip + i] : 0);
  return v;
}

// a before b in the merge (InternalKeyComparator order), given their user-key
// prefixes: the prefixes decide unless equal.
__device__ __forceinline__ bool entry_le(const JobDev& J, uint32_t a, uint64_t pa, uint32_t b,
                                         uint64_t pb) {
  if (pa != pb) return pa < pb;
  return ikey_cmp(J.keys + J.e_koff[a], J.e_klen[a], J.keys + J.e_koff[b], J.e_klen[b]) <= 0;
}

// Same user key?  (pa, pb: their user-key prefixes)
__device__ __forceinline__ bool same_user_key(const JobDev& J, uint32_t a, uint64_t pa, uint32_t b,
                                              uint64_t pb) {
  if (pa != pb) return false;
  uint32_t al = J.e_klen[a] - 8, bl = J.e_klen[b] - 8;
  if (al != bl) return false;
  const uint8_t* x = J.keys + J.e_koff[a];
  const uint8_t* y = J.keys + J.e_koff[b];
  for (uint32_t i = 0; i < al; i++)
    if (x[i] != y[i]) return false;
  return true;
}

// Hash of util/hash.cc:22-51 (the bloom filter's hash) over bytes that may
// start at any alignment, four at a time from aligned word loads realigned by
// funnel shifts.  Reads up to one word past the data: only for data in a
// buffer with that much slack (the key arena keeps 16 bytes).
__device__ __forceinline__ uint32_t leveldb_hash_words(const uint8_t* data, uint32_t n,
                                                       uint32_t seed) {
  const uint32_t m = 0xc6a4a793u;
  const uintptr_t a = reinterpret_cast<uintptr_t>(data);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = 8 * (uint32_t)(a & 3);
  uint32_t h = seed ^ (n * m);
  uint32_t lo = q[0], i = 0;
  for (; i + 4 <= n; i += 4) {
    const uint32_t hi = q[(i >> 2) + 1];
    h += __funnelshift_r(lo, hi, sh);
    lo = hi;
    h *= m;
    h ^= (h >> 16);
  }
  const uint32_t r = n - i;
  if (r) {
    const uint32_t w = __funnelshift_r(lo, q[(i >> 2) + 1], sh);  // bytes i.. of the data
    h += w & ((1u << (8 * r)) - 1u);
    h *= m;
    h ^= (h >> 24);
  }
  return h;
}

// a % d for 32-bit a and a divisor d >= 1 fixed over many calls, from
// M = floor((2^64 - 1) / d) + 1: (M a mod 2^64) d >> 64 (Lemire, Kaser and
// Kurz, "Faster remainder by direct computation", 2019).
struct FastMod {
  uint64_t M;
  uint32_t d;
  __device__ __forceinline__ explicit FastMod(uint32_t div) : M(~0ull / div + 1), d(div) {}
  __device__ __forceinline__ uint32_t operator()(uint32_t a) const {
    return (uint32_t)__umul64hi(M * a, d);
  }
};

// ---------------------------------------------------------------------------
// CRC32C

// Fills a 256-entry byte table in shared memory (call with all threads, then
// __syncthreads()).
__device__ __forceinline__ void crc_table_init(uint32_t* tab) {
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = i;
#pragma unroll
    for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
    tab[i] = c;
  }
}

// Raw CRC register update (no inversion) over n bytes.
__device__ __forceinline__ uint32_t crc_raw(const uint32_t* tab, uint32_t c, const uint8_t* p,
                                            uint32_t n) {
  for (uint32_t i = 0; i < n; i++) c = tab[(c ^ p[i]) & 0xff] ^ (c >> 8);
  return c;
}

// a * b mod P with the byte table tab (tab[i] = register after byte i from
// 0, that is i * x^32 mod P): a's four bytes by Horner, the byte groups of
// b x^j (j < 8) by their bits, and each step of x^8 as one zero byte fed to
// the register.
__device__ __forceinline__ uint32_t gf2_mulmod_tab(const uint32_t* __restrict__ tab, uint32_t a,
                                                   uint32_t b) {
  uint32_t bx[8];
  bx[0] = b;
#pragma unroll
  for (int j = 1; j < 8; j++) bx[j] = (bx[j - 1] >> 1) ^ ((bx[j - 1] & 1) ? kCrcPoly : 0u);
  // reflected: bits 31..24 of a are x^0..x^7, bits 7..0 are x^24..x^31
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (k) r = tab[r & 0xff] ^ (r >> 8);  // r x^8
    const uint32_t byte = (a >> (8 * k)) & 0xff;  // degrees 8(3-k) .. 8(3-k)+7
#pragma unroll
    for (int d = 0; d < 8; d++)
      if (byte & (0x80u >> d)) r ^= bx[d];  // bit 7 - d of the byte: x^d of its group
  }
  return r;
}

// a * b mod P in the reflected representation (bit 31 = x^0).
__host__ __device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
  uint32_t p = 0;
  for (int i = 0; i < 32; i++) {
    if (a & 0x80000000u) p ^= b;
    a <<= 1;
    b = (b & 1) ? (b >> 1) ^ kCrcPoly : (b >> 1);
  }
  return p;
}

// x^(8n) mod P: table lookup for small n, square-and-multiply from the table
// entries x^(8*2^k) beyond it.
__device__ __forceinline__ uint32_t crc_xpow8(const JobDev& J, uint64_t n) {
  const uint64_t N = J.crc_xpow_n;
  if (n < N) return J.crc_xpow[n];
  // n = q*N + r:  x^(8n) = (x^(8N))^q * x^(8r), the power by squaring.
  uint32_t r = J.crc_xpow[n % N];
  uint64_t q = n / N;
  uint32_t base = gf2_mulmod(J.crc_xpow[N - 1], J.crc_xpow[1]);  // x^(8N)
  while (q) {
    if (q & 1) r = gf2_mulmod(r, base);
    base = gf2_mulmod(base, base);
    q >>= 1;
  }
  return r;
}

// shift(c, n): the raw CRC register after feeding n zero bytes.
__device__ __forceinline__ uint32_t crc_shift(const JobDev& J, uint32_t c, uint64_t n) {
  return gf2_mulmod(crc_xpow8(J, n), c);
}

// shift(c, n) with the byte table tab (in shared memory): x^(8n) as the
// product of two table entries (n = hi N + lo, N = crc_xpow_n) for n < N^2,
// then one more product with c.
__device__ __forceinline__ uint32_t crc_shift_tab(const JobDev& J, const uint32_t* tab,
                                                  uint32_t c, uint64_t n) {
  const uint64_t N = J.crc_xpow_n;
  if (n >= N * N) return crc_shift(J, c, n);
  const uint32_t lo = (uint32_t)(n % N), hi = (uint32_t)(n / N);
  uint32_t m = __ldg(J.crc_xpow + lo);
  if (hi) m = gf2_mulmod_tab(tab, m, __ldg(J.crc_xpow_hi + hi));
  return gf2_mulmod_tab(tab, c, m);
}

// Masked CRC32C of contents followed by the type byte: the block trailer of
// table/table_builder.cc:186-189, computed cooperatively by one warp over `n`
// bytes at `p` (the type byte, 0 for an uncompressed block, is appended
// implicitly).
__device__ __forceinline__ uint32_t warp_block_crc(const JobDev& J, const uint32_t* tab,
                                                   const uint8_t* p, uint32_t n,
                                                   uint8_t type = 0) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t total = n + 1;  // contents + type byte
  uint32_t seg = (total + 31) / 32;
  uint32_t b = lane * seg;
  uint32_t e = min(total, b + seg);
  uint32_t c = 0;
  for (uint32_t i = b; i < e; i++) {
    uint8_t byte = i < n ? p[i] : type;
    c = tab[(c ^ byte) & 0xff] ^ (c >> 8);
  }
  // shift each lane's raw CRC by the bytes after its segment, xor together
  uint32_t after = total > e ? total - e : 0;
  uint32_t v = (b < total) ? crc_shift(J, c, after) : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, o);
  // init 0xffffffff contributes shift(~0, total); final inversion
  uint32_t full = v ^ crc_shift(J, 0xffffffffu, total) ^ 0xffffffffu;
  return ((full >> 15) | (full << 17)) + 0xa282ead8u;  // crc32c::Mask
}

// Up to kMax (a multiple of 4, at most 32) bytes from src (any alignment) to
// dst: every word that holds a needed byte is loaded before any byte is
// stored (no load waits on the previous store), then the words are realigned
// by funnel shifts.
template <uint32_t kMax = 32>
__device__ __forceinline__ void copy_small(uint8_t* dst, const uint8_t* src, uint32_t len) {
  if (!len) return;
  constexpr uint32_t kW = kMax / 4 + 1;
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uint32_t* base = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = 8 * (uint32_t)(a & 3);
  const uint32_t nw = ((uint32_t)(a & 3) + len + 3) >> 2;  // words holding the bytes
  uint32_t w[kW];
#pragma unroll
  for (uint32_t i = 0; i < kW; i++) w[i] = i < nw ? __ldg(base + i) : 0u;
  uint32_t r[kW - 1];
#pragma unroll
  for (uint32_t i = 0; i + 1 < kW; i++) r[i] = __funnelshift_r(w[i], w[i + 1], sh);
#pragma unroll
  for (uint32_t i = 0; i < kMax; i++)
    if (i < len) dst[i] = (uint8_t)(r[i >> 2] >> (8 * (i & 3)));
}

// Up to 32 bytes from src (global memory, any alignment) to dst (shared
// memory, any alignment): the destination's whole words with word stores,
// its partial words at both ends byte by byte (their other bytes belong to
// other writers).  Only source words that hold a needed byte are loaded.
__device__ __forceinline__ void copy_small_w(uint8_t* dst, const uint8_t* src, uint32_t len) {
  if (!len) return;
  const uintptr_t d = reinterpret_cast<uintptr_t>(dst), s = reinterpret_cast<uintptr_t>(src);
  const uint32_t da = (uint32_t)(d & 3);
  // destination word q covers source bytes from s - da + 4q
  const uintptr_t s0 = s - da;
  const uint32_t* base = reinterpret_cast<const uint32_t*>(s0 & ~uintptr_t(3));
  const uint32_t sh = 8 * (uint32_t)(s0 & 3);
  const uintptr_t b0 = reinterpret_cast<uintptr_t>(base);
  uint32_t w[11];
#pragma unroll
  for (uint32_t i = 0; i < 11; i++) {
    const uintptr_t wa = b0 + 4 * i;  // word [wa, wa + 4) holds a needed byte?
    w[i] = (wa + 4 > s && wa < s + len) ? __ldg(base + i) : 0u;
  }
  uint32_t* dw = reinterpret_cast<uint32_t*>(d - da);
  const uint32_t end = da + len;  // destination bytes [da, end) of the words from dw
#pragma unroll
  for (uint32_t q = 0; q < 9; q++) {
    if (4 * q >= end) break;
    const uint32_t v = __funnelshift_r(w[q], w[q + 1], sh);
    if (4 * q >= da && 4 * q + 4 <= end) {
      dw[q] = v;
    } else {
      uint8_t* db = reinterpret_cast<uint8_t*>(dw + q);
#pragma unroll
      for (uint32_t i = 0; i < 4; i++)
        if (4 * q + i >= da && 4 * q + i < end) db[i] = (uint8_t)(v >> (8 * i));
    }
  }
}

// The job descriptor into shared memory (all threads of the CTA; a
// __syncthreads() must follow): kernels that stream large arrays through L1
// read their descriptor's fields from there instead of reloading evicted
// lines from L2.
__device__ __forceinline__ void copy_job(const JobDev* __restrict__ src, JobDev* dst) {
  static_assert(sizeof(JobDev) % 8 == 0, "JobDev is copied in 8-byte words");
  const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
  uint64_t* d = reinterpret_cast<uint64_t*>(dst);
  for (uint32_t i = threadIdx.x; i < sizeof(JobDev) / 8; i += blockDim.x) d[i] = s[i];
}

// Error reporting: the first error code wins.
__device__ __forceinline__ void set_error(Counters* c, uint32_t code, uint32_t detail) {
  if (atomicCAS(&c->error, 0u, code) == 0u) c->error_detail = detail;
}

}  // namespace lc

namespace lc {

// ---------------------------------------------------------------------------
// Asynchronous 16-byte global -> shared copies (cp.async, LDGSTS): many in
// flight per warp without holding registers; completion by wait_all.

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Slicing-by-4 CRC32C tables in shared memory: tab4[k][x] is the register
// update for byte x followed by k zero bytes (tab4[0] is the byte table).
__device__ __forceinline__ void crc_tables4_init(uint32_t* tab4) {
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = i;
#pragma unroll
    for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
    tab4[i] = c;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = tab4[i];
    for (int k = 1; k < 4; k++) {
      c = (c >> 8) ^ tab4[c & 0xff];
      tab4[256 * k + i] = c;
    }
  }
}

// Raw CRC register update over [p, p+n) in shared memory, four bytes per
// step once p is word aligned.
__device__ __forceinline__ uint32_t crc_raw4(const uint32_t* tab4, uint32_t c, const uint8_t* p,
                                             uint32_t n) {
  uint32_t i = 0;
  while (i < n && (reinterpret_cast<uintptr_t>(p + i) & 3)) {
    c = tab4[(c ^ p[i]) & 0xff] ^ (c >> 8);
    i++;
  }
  for (; i + 4 <= n; i += 4) {
    c ^= *reinterpret_cast<const uint32_t*>(p + i);
    c = tab4[768 + (c & 0xff)] ^ tab4[512 + ((c >> 8) & 0xff)] ^ tab4[256 + ((c >> 16) & 0xff)] ^
        tab4[c >> 24];
  }
  for (; i < n; i++) c = tab4[(c ^ p[i]) & 0xff] ^ (c >> 8);
  return c;
}

// ---------------------------------------------------------------------------
// Block CRC32C over 16-byte chunks, lane l of a warp taking chunks l, l + 32,
// l + 64, ... (one 512-byte row of the block per step of all 32 lanes).
//
// The raw register after n bytes is linear in the bytes and in the register
// it started from, and a register u before 16 bytes x equals register 0
// before x with u xored into its first four bytes.  So a lane keeps
//   u <- H(x ^ u),  H(x) = register after x and 496 zero bytes, from 0,
// which accounts for the other lanes' bytes of the row as zeros; the block's
// register is the xor over the lanes of their u, each moved back (x^-8n) by
// the bytes it was carried past the block's end.  H is linear in the 128 bits
// of x: the xor of one lookup per kCrcFieldBits-bit field, each in its own
// table.  The CRC's initial all-ones register is the same as ones xored into
// the block's first four bytes.
constexpr uint32_t kCrcFieldBits = 5;
constexpr uint32_t kCrcFields = (128 + kCrcFieldBits - 1) / kCrcFieldBits;
constexpr uint32_t kCrcFieldEntries = 1u << kCrcFieldBits;
constexpr uint32_t kCrcH5Words = kCrcFields * kCrcFieldEntries;  // the row tables
constexpr uint32_t kCrcRowBytes = 512;   // 32 lanes x 16 bytes
constexpr uint32_t kCrcXinvN = 512;      // back shifts of 0..511 bytes
// The back shifts' shared-memory copy skips a word after every 16 entries:
// a warp's lanes index it 16 apart (one lane per 16-byte chunk column), which
// in a dense copy falls on two banks.
constexpr uint32_t kCrcXinvSmem = kCrcXinvN + kCrcXinvN / 16;
__host__ __device__ __forceinline__ uint32_t xinv_slot(uint32_t n) { return n + (n >> 4); }

// H(w0..w3) from the row tables (table i at h5[kCrcFieldEntries i], indexed
// by bits [W i, W i + W) of the little-endian 128-bit chunk); the field's
// byte offset into its table comes from one shift and one mask.
__device__ __forceinline__ uint32_t crc_h5(const uint32_t* __restrict__ h5, uint32_t w0,
                                           uint32_t w1, uint32_t w2, uint32_t w3) {
  const uint32_t w[5] = {w0, w1, w2, w3, 0u};
  constexpr uint32_t mask = (kCrcFieldEntries - 1) << 2;
  const uint8_t* t = reinterpret_cast<const uint8_t*>(h5);
  uint32_t r = 0;
#pragma unroll
  for (uint32_t i = 0; i < kCrcFields; i++) {
    const uint32_t s = kCrcFieldBits * i, q = s >> 5, o = s & 31;
    uint32_t f4;
    if (o + kCrcFieldBits <= 32)
      f4 = (o >= 2 ? (w[q] >> (o - 2)) : (w[q] << (2 - o))) & mask;
    else
      f4 = __funnelshift_r(w[q], w[q + 1], o - 2) & mask;
    r ^= *reinterpret_cast<const uint32_t*>(t + 4 * kCrcFieldEntries * i + f4);
  }
  return r;
}

// The bytes of word x at grid position pos that belong to the message
// [m0, m1), zero elsewhere, with the grid bytes [i0, i0 + 4) inverted (the
// message's first four when it starts the CRC: the initial register).
__device__ __forceinline__ uint32_t crc_edge_word(uint32_t x, uint32_t pos, uint32_t m0,
                                                  uint32_t m1, uint32_t i0) {
  const auto lo_mask = [](int32_t k) -> uint32_t {  // bytes [0, k) of a word, k clamped to 0..4
    return k <= 0 ? 0u : (k >= 4 ? 0xffffffffu : (1u << (8 * k)) - 1u);
  };
  const int32_t a = (int32_t)m0 - (int32_t)pos, b = (int32_t)m1 - (int32_t)pos;
  const int32_t c = (int32_t)i0 - (int32_t)pos;
  const uint32_t keep = lo_mask(b) & ~lo_mask(a);
  const uint32_t inv = lo_mask(c + 4) & ~lo_mask(c);
  return (x & keep) ^ inv;
}

// One lane's chunk at grid position p (16-aligned) into its CRC register u,
// for the message [m0, m1) of the grid (init: the message starts the CRC, so
// its first four bytes are inverted).
__device__ __forceinline__ uint32_t crc_chunk_step(const uint32_t* __restrict__ h5, uint32_t u,
                                                   uint32_t p, uint32_t m0, uint32_t m1,
                                                   uint32_t w0, uint32_t w1, uint32_t w2,
                                                   uint32_t w3, bool init = true) {
  if (p < m0 + 4 || p + 16 > m1) {
    const uint32_t i0 = init ? m0 : 0x40000000u;  // far past any chunk: nothing inverted
    w0 = crc_edge_word(w0, p, m0, m1, i0);
    w1 = crc_edge_word(w1, p + 4, m0, m1, i0);
    w2 = crc_edge_word(w2, p + 8, m0, m1, i0);
    w3 = crc_edge_word(w3, p + 12, m0, m1, i0);
  }
  return crc_h5(h5, w0 ^ u, w1, w2, w3);
}

// The raw register at the message's end from the lanes' registers (lane l's
// last chunk at grid position `last`, 0xffffffff when it had none), the same
// in every lane.  xinv is the back shifts' padded shared-memory copy
// (xinv_slot).
__device__ __forceinline__ uint32_t crc_rows_raw(const uint32_t* __restrict__ xinv,
                                                 const uint32_t* __restrict__ tab8, uint32_t u,
                                                 uint32_t last, uint32_t m1) {
  uint32_t v = 0;
  if (last != 0xffffffffu) v = gf2_mulmod_tab(tab8, u, xinv[xinv_slot(last + kCrcRowBytes - m1)]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The masked CRC from the lanes' registers: lane l's last chunk was at grid
// position `last` (0xffffffff when it had none) and the message ends at m1.
__device__ __forceinline__ uint32_t crc_rows_finish(const uint32_t* __restrict__ xinv,
                                                    const uint32_t* __restrict__ tab8, uint32_t u,
                                                    uint32_t last, uint32_t m1) {
  const uint32_t full = crc_rows_raw(xinv, tab8, u, last, m1) ^ 0xffffffffu;
  return ((full >> 15) | (full << 17)) + 0xa282ead8u;  // crc32c::Mask
}

// Masked block trailer CRC of the block [p, p + n) plus the zero type byte at
// p[n], read from memory in 16-byte chunks by one warp (p - (p & 15) is the
// grid origin; bytes of the chunks outside the block are read and ignored).
__device__ __forceinline__ uint32_t warp_block_crc_rows(const uint32_t* __restrict__ h5,
                                                        const uint32_t* __restrict__ xinv,
                                                        const uint32_t* __restrict__ tab8,
                                                        const uint8_t* p, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t m0 = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 15), m1 = m0 + n + 1;
  const uint8_t* g = p - m0;
  uint32_t u = 0, last = 0xffffffffu;
  for (uint32_t q = 16 * lane; q < m1; q += kCrcRowBytes) {
    const uint4 x = __ldcg(reinterpret_cast<const uint4*>(g + q));  // the warp's own stores, via L2
    u = crc_chunk_step(h5, u, q, m0, m1, x.x, x.y, x.z, x.w);
    last = q;
  }
  return crc_rows_finish(xinv, tab8, u, last, m1);
}

}  // namespace lc
