// Decode: input tables -> entries (keys reconstructed into a key arena, values
// left in place).
//
// Follows the reference's table reader: Footer::DecodeFrom
// (table/format.cc:42-62), the index block's block handles
// (table/table.cc:38-111), and Block::Iter's entry parse (table/block.cc:
// 170-190, 340-367).  The LUDA restart word (table/block_builder.cc:62-66,
// 90-96) is (offset << 8) | entries in that restart run, so every restart run
// is decoded independently: the run's first entry has no shared prefix, and
// the run's entry count is known from the word before any entry is parsed.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "lc_device.cuh"
#include "lc_kernels.h"

namespace lc {

namespace {

constexpr uint32_t kMagicLo = 0x8b80fb57u;  // kTableMagicNumber (table/format.h:77)
constexpr uint32_t kMagicHi = 0xdb477524u;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_excl(T v, T* total) {
  const int lane = threadIdx.x & 31;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += u;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

// Locates the index block of a table; false if the footer is invalid.
__device__ bool parse_footer(const uint8_t* t, uint64_t n, uint64_t* i_off, uint64_t* i_size) {
  if (n < kFooter) return false;
  const uint8_t* f = t + n - kFooter;
  if (ld_le32(f + 40) != kMagicLo || ld_le32(f + 44) != kMagicHi) return false;
  uint64_t m_off, m_size;
  const uint8_t* p = f;
  const uint8_t* lim = f + 40;
  if (!(p = get_varint64(p, lim, &m_off))) return false;
  if (!(p = get_varint64(p, lim, &m_size))) return false;
  if (!(p = get_varint64(p, lim, i_off))) return false;
  if (!(p = get_varint64(p, lim, i_size))) return false;
  if (*i_off > n || *i_size < 4 || *i_size + kTrailer > n - *i_off) return false;
  return true;
}

// Parses one entry header at p (bounded by lim).  Returns the key-delta
// pointer or nullptr.
__device__ __forceinline__ const uint8_t* entry_header(const uint8_t* p, const uint8_t* lim,
                                                       uint32_t* shared, uint32_t* non_shared,
                                                       uint32_t* vlen) {
  if (lim - p < 3) return nullptr;
  uint32_t a = p[0], b = p[1], c = p[2];
  if ((a | b | c) < 128) {
    *shared = a;
    *non_shared = b;
    *vlen = c;
    p += 3;
  } else {
    if (!(p = get_varint32(p, lim, shared))) return nullptr;
    if (!(p = get_varint32(p, lim, non_shared))) return nullptr;
    if (!(p = get_varint32(p, lim, vlen))) return nullptr;
  }
  if ((uint64_t)(lim - p) < (uint64_t)*non_shared + *vlen) return nullptr;
  return p;
}

__global__ void k_table_index_count(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  const uint32_t t = blockIdx.x;
  if (t >= J.n_tables) return;
  const TableDesc T = J.tables[t];
  if (T.cached) {  // read from its decoded form: pseudo blocks of kDecRunBlock entries
    if (threadIdx.x == 0)
      J.tbl_nblocks[t] = (uint32_t)((J.dec_runs[t].n + kDecRunBlock - 1) / kDecRunBlock);
    return;
  }
  const uint8_t* base = J.in + T.off;
  __shared__ uint64_t s_ioff, s_isize;
  __shared__ uint32_t s_nr, s_ok;
  __shared__ uint32_t s_part[32];
  if (threadIdx.x == 0) {
    uint64_t io = 0, is = 0;
    bool ok = parse_footer(base, T.size, &io, &is);
    uint32_t nr = 0;
    if (ok) {
      nr = ld_le32(base + io + is - 4);
      if ((uint64_t)nr * 4 + 4 > is) ok = false;
    }
    if (!ok) set_error(J.ctr, kErrBadFooter, t);
    s_ioff = io;
    s_isize = is;
    s_nr = nr;
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) {
    if (threadIdx.x == 0) J.tbl_nblocks[t] = 0;
    return;
  }
  const uint8_t* ra = base + s_ioff + s_isize - 4 - 4ull * s_nr;
  uint32_t sum = 0;
  for (uint32_t r = threadIdx.x; r < s_nr; r += blockDim.x) sum += ld_le32(ra + 4ull * r) & 0xff;
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; w++) s += s_part[w];
    J.tbl_nblocks[t] = s;
  }
}

__global__ void k_table_index_entries(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  const uint32_t t = blockIdx.x;
  if (t >= J.n_tables) return;
  const TableDesc T = J.tables[t];
  if (T.cached) {
    const uint64_t out_base = J.tbl_block_base[t], out_end = J.tbl_block_base[t + 1];
    for (uint64_t o = out_base + threadIdx.x; o < out_end && o < J.cap_blocks_in; o += blockDim.x) {
      J.blk_off[o] = ((uint64_t)t << 32) | ((o - out_base) * kDecRunBlock);
      J.blk_size[o] = kPseudoBlock;
      J.blk_run[o] = T.run;
    }
    return;
  }
  const uint8_t* base = J.in + T.off;
  uint64_t io, is;
  if (!parse_footer(base, T.size, &io, &is)) return;  // error already recorded
  const uint32_t nr = ld_le32(base + io + is - 4);
  if ((uint64_t)nr * 4 + 4 > is) return;
  const uint8_t* idx = base + io;
  const uint64_t ra_off = is - 4 - 4ull * nr;
  const uint8_t* ra = idx + ra_off;
  const uint64_t out_base = J.tbl_block_base[t];
  const uint64_t out_end = J.tbl_block_base[t + 1];
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base_r = 0; base_r < nr; base_r += blockDim.x) {
    const uint32_t r = base_r + threadIdx.x;
    uint32_t w = r < nr ? ld_le32(ra + 4ull * r) : 0;
    uint32_t cnt = w & 0xff;
    // block-wide exclusive scan of cnt
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t tot;
    uint32_t ex = warp_excl(cnt, &tot);
    if (lane == 0) s_warp[wid] = tot;
    __syncthreads();
    uint32_t before = s_carry;
    for (int k = 0; k < wid; k++) before += s_warp[k];
    uint32_t all = 0;
    for (int k = 0; k < (int)((blockDim.x + 31) / 32); k++) all += s_warp[k];
    ex += before;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += all;
    if (r < nr) {
      uint64_t start = w >> 8;
      uint64_t end = (r + 1 < nr) ? (ld_le32(ra + 4ull * (r + 1)) >> 8) : ra_off;
      bool ok = start <= end && end <= ra_off;
      const uint8_t* p = idx + start;
      const uint8_t* lim = idx + end;
      for (uint32_t k = 0; ok && k < cnt; k++) {
        uint32_t sh, ns, vl;
        const uint8_t* q = entry_header(p, lim, &sh, &ns, &vl);
        if (!q) {
          ok = false;
          break;
        }
        q += ns;
        uint64_t b_off, b_size;
        const uint8_t* h = q;
        if (!(h = get_varint64(h, q + vl, &b_off)) || !(h = get_varint64(h, q + vl, &b_size))) {
          ok = false;
          break;
        }
        if (b_off > T.size || b_size + kTrailer > T.size - b_off) {
          ok = false;
          break;
        }
        const uint64_t o = out_base + ex + k;
        if (o >= out_end || o >= J.cap_blocks_in) {
          ok = false;
          break;
        }
        J.blk_off[o] = T.off + b_off;
        J.blk_size[o] = (uint32_t)b_size;
        J.blk_run[o] = T.run;
        p = q + vl;
      }
      if (ok && p != lim) ok = false;
      if (!ok) set_error(J.ctr, kErrBadIndex, t);
    }
    __syncthreads();
  }
}

// A pseudo block: entries [*j0, *j1) of the decoded run of table *t.
__device__ __forceinline__ const DecRun& pseudo_block(const JobDev& J, uint64_t b, uint32_t* t,
                                                      uint64_t* j0, uint64_t* j1) {
  const uint64_t o = J.blk_off[b];
  *t = (uint32_t)(o >> 32);
  const DecRun& R = J.dec_runs[*t];
  *j0 = o & 0xffffffffull;
  *j1 = min(R.n, *j0 + kDecRunBlock);
  return R;
}

// Entry descriptors of a pseudo block (key lengths, value places and
// lengths); its key bytes, one lane per entry.  Returns the key bytes and
// the longest key; false if a key is shorter than 8 bytes or a value lies
// outside its table.
__device__ __forceinline__ bool pseudo_entries(const JobDev& J, uint64_t b, uint64_t ebase,
                                               uint32_t lane, uint32_t lanes, uint64_t* kbytes,
                                               uint32_t* maxk) {
  uint32_t t;
  uint64_t j0, j1;
  const DecRun& R = pseudo_block(J, b, &t, &j0, &j1);
  const TableDesc T = J.tables[t];
  bool ok = true;
  uint32_t mk = 0;
  for (uint64_t j = j0 + lane; j < j1; j += lanes) {
    const uint64_t e = ebase + (j - j0);
    const uint32_t kl = (uint32_t)(R.kcum[j + 1] - R.kcum[j]);
    const uint32_t vl = R.vlen[j], vp = R.vpos[j];
    if (kl < 8 || (uint64_t)vp + vl > T.size || e >= J.cap_entries) {
      ok = false;
      continue;
    }
    J.e_klen[e] = kl;
    J.e_vlen[e] = vl;
    J.e_voff[e] = (uint32_t)(T.off + vp);
    mk = max(mk, kl);
  }
  *kbytes = R.kcum[j1] - R.kcum[j0];
  *maxk = mk;
  return ok;
}

// Key bytes (one contiguous copy), key offsets, prefixes and tags of a
// pseudo block, by one warp; its keys start at kbase in the arena.
__device__ __forceinline__ void pseudo_keys(const JobDev& J, uint64_t b, uint64_t ebase,
                                            uint64_t kbase, uint32_t lane) {
  uint32_t t;
  uint64_t j0, j1;
  const DecRun& R = pseudo_block(J, b, &t, &j0, &j1);
  const uint64_t k0 = R.kcum[j0], kn = R.kcum[j1] - k0;
  const uint8_t* src = R.keys + k0;
  uint8_t* dst = J.keys + kbase;
  for (uint64_t x = lane; x < kn; x += 32) dst[x] = src[x];
  for (uint64_t j = j0 + lane; j < j1; j += 32) {
    const uint64_t e = ebase + (j - j0);
    J.e_koff[e] = (uint32_t)(kbase + (R.kcum[j] - k0));
    J.e_pfx[e] = R.pfx[j];
    J.e_tag[e] = R.tag[j];
  }
}

// Walks the entries of one restart run without writing them: counts key bytes
// and validates every header against the run's bounds.
__device__ __forceinline__ bool walk_run(const uint8_t* p, const uint8_t* lim, uint32_t cnt,
                                         uint64_t* kbytes, uint32_t* maxk, bool* short_key) {
  uint32_t prev = 0;
  uint64_t kb = 0;
  for (uint32_t k = 0; k < cnt; k++) {
    uint32_t sh, ns, vl;
    const uint8_t* q = entry_header(p, lim, &sh, &ns, &vl);
    if (!q) return false;
    if ((k == 0 && sh != 0) || sh > prev) return false;
    uint32_t kl = sh + ns;
    if (kl < 8) *short_key = true;
    kb += kl;
    *maxk = max(*maxk, kl);
    prev = kl;
    p = q + ns + vl;
  }
  *kbytes = kb;
  return p == lim;
}

struct BlockView {
  const uint8_t* p;
  uint64_t ra;  // offset of the restart array (end of entries)
  uint32_t nr;
  bool ok;
};

// View of data block b whose bytes are at `base` (a shared-memory stage or
// the block in global memory).
__device__ __forceinline__ BlockView block_view(const JobDev& J, uint64_t b, const uint8_t* base) {
  BlockView v;
  v.p = base;
  const uint32_t size = J.blk_size[b];
  v.ok = size >= 4;
  v.nr = v.ok ? ld_le32(v.p + size - 4) : 0;
  if (v.ok && (uint64_t)v.nr * 4 + 4 > size) v.ok = false;
  v.ra = v.ok ? size - 4 - 4ull * v.nr : 0;
  return v;
}

__device__ __forceinline__ void run_bounds(const BlockView& v, uint32_t r, uint64_t* start,
                                           uint64_t* end, uint32_t* cnt) {
  const uint32_t w = ld_le32(v.p + v.ra + 4ull * r);
  *cnt = w & 0xff;
  *start = w >> 8;
  *end = (r + 1 < v.nr) ? (ld_le32(v.p + v.ra + 4ull * (r + 1)) >> 8) : v.ra;
}

// Per-warp shared memory of the staged decode kernels.
constexpr uint32_t kDecWarps = 4;
constexpr uint32_t kDecStage = 8448;    // data block bytes + 16-byte phase
constexpr uint32_t kDecMaxEnt = 512;    // entries of one staged block
constexpr uint32_t kDecKeyBuf = 32 * 132 + 32;  // 4 KiB of keys, or 32 lane slices of 132 bytes
constexpr uint32_t kDecLastKey = 256;   // longest key the staged path rebuilds
struct DecWarpSmem {
  uint8_t stage[kDecStage];
  uint8_t keybuf[kDecKeyBuf];
  uint16_t dpos[kDecMaxEnt];  // key delta position in the stage
  uint16_t sh[kDecMaxEnt];    // shared prefix
  uint16_t kl[kDecMaxEnt];    // key length
  uint16_t vl[kDecMaxEnt];    // value length
  uint8_t lastkey[kDecLastKey];  // last key of the previous group of 32 entries
};

// Copies data block b into this warp's stage at the block's own 16-byte phase
// with 16-byte loads; returns the staged pointer, or nullptr if it is too big.
__device__ __forceinline__ const uint8_t* stage_block(const JobDev& J, uint64_t b, uint8_t* stage,
                                                      uint32_t lane) {
  const uint8_t* src = J.in + J.blk_off[b];
  const uint32_t size = J.blk_size[b];
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uint32_t phase = (uint32_t)(a & 15);
  if (size + phase + 16 > kDecStage) return nullptr;
  const uintptr_t base = a - phase;
  const uint32_t nch = (phase + size + 15) >> 4;
  const uintptr_t lo = reinterpret_cast<uintptr_t>(J.in), hi = reinterpret_cast<uintptr_t>(J.in_end);
  for (uint32_t c = lane; c < nch; c += 32) {
    const uintptr_t q = base + 16ull * c;
    if (q >= lo && q + 16 <= hi) {
      cp_async16(stage + 16 * c, reinterpret_cast<const void*>(q));
    } else {
      uint32_t w[4] = {0, 0, 0, 0};
      for (int i = 0; i < 16; i++) {
        const uintptr_t x = q + i;
        if (x >= a && x < a + size) w[i >> 2] |= (uint32_t)(*reinterpret_cast<const uint8_t*>(x)) << (8 * (i & 3));
      }
      *reinterpret_cast<uint4*>(stage + 16 * c) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
  cp_async_wait_all();
  __syncwarp();
  return stage + phase;
}

__device__ void block_count_one(const JobDev& J, uint64_t b, uint32_t lane, const uint8_t* base) {
  BlockView v = block_view(J, b, base);
  uint64_t ent = 0, kb = 0;
  uint32_t maxk = 0;
  bool ok = v.ok, short_key = false;
  for (uint32_t r = lane; ok && r < v.nr; r += 32) {
    uint64_t s, e;
    uint32_t cnt;
    run_bounds(v, r, &s, &e, &cnt);
    if (s > e || e > v.ra) {
      ok = false;
      break;
    }
    uint64_t rk = 0;
    if (!walk_run(v.p + s, v.p + e, cnt, &rk, &maxk, &short_key)) {
      ok = false;
      break;
    }
    ent += cnt;
    kb += rk;
  }
  const bool all_ok = __all_sync(0xffffffffu, ok);
  const bool any_short = __any_sync(0xffffffffu, short_key);
  ent = warp_sum(ent);
  kb = warp_sum(kb);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
  if (lane == 0) {
    if (!all_ok) set_error(J.ctr, kErrBadBlock, (uint32_t)b);
    else if (any_short) set_error(J.ctr, kErrShortKey, (uint32_t)b);
    J.blk_nent[b] = all_ok ? (uint32_t)ent : 0;
    J.blk_kbytes[b] = all_ok ? kb : 0;
    atomicMax(&J.ctr->max_klen, maxk);
  }
}

__global__ void __launch_bounds__(kDecWarps * 32) k_block_count(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  extern __shared__ __align__(16) uint8_t dec_smem[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  DecWarpSmem& W = reinterpret_cast<DecWarpSmem*>(dec_smem)[warp];
  // after a footer or index error some block handles were never written
  if (J.ctr->error) return;
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  for (uint64_t b = (uint64_t)blockIdx.x * kDecWarps + warp; b < nblk;
       b += (uint64_t)gridDim.x * kDecWarps) {
    if (J.blk_size[b] == kPseudoBlock) {
      uint32_t t;
      uint64_t j0, j1;
      const DecRun& R = pseudo_block(J, b, &t, &j0, &j1);
      uint32_t mk = 0;
      for (uint64_t j = j0 + lane; j < j1; j += 32) mk = max(mk, (uint32_t)(R.kcum[j + 1] - R.kcum[j]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mk = max(mk, __shfl_xor_sync(0xffffffffu, mk, o));
      if (lane == 0) {
        J.blk_nent[b] = (uint32_t)(j1 - j0);
        J.blk_kbytes[b] = R.kcum[j1] - R.kcum[j0];
        atomicMax(&J.ctr->max_klen, mk);
      }
      continue;
    }
    const uint8_t* st = stage_block(J, b, W.stage, lane);
    block_count_one(J, b, lane, st ? st : J.in + J.blk_off[b]);
    __syncwarp();
  }
}

// Entries per data block from its restart array alone (the LUDA restart word
// holds the entry count of its run): one thread per block.  The run byte
// ranges are checked here; the entries themselves when they are decoded.
__global__ void k_block_restarts(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // after a footer or index error some handles are unset
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblk;
       b += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t size = J.blk_size[b];
    if (size == kPseudoBlock) {
      uint32_t t;
      uint64_t j0, j1;
      pseudo_block(J, b, &t, &j0, &j1);
      J.blk_nent[b] = (uint32_t)(j1 - j0);
      continue;
    }
    const uint8_t* p = J.in + J.blk_off[b];
    bool ok = size >= 4;
    const uint32_t nr = ok ? ld_le32(p + size - 4) : 0;
    if (ok && (uint64_t)nr * 4 + 4 > size) ok = false;
    const uint64_t ra = ok ? size - 4 - 4ull * nr : 0;
    uint64_t ent = 0, prev_end = 0;
    for (uint32_t r = 0; ok && r < nr; r++) {
      const uint32_t w = ld_le32(p + ra + 4ull * r);
      const uint64_t s0 = w >> 8;
      const uint64_t e0 = (r + 1 < nr) ? (ld_le32(p + ra + 4ull * (r + 1)) >> 8) : ra;
      if (s0 > e0 || e0 > ra || s0 < prev_end) ok = false;
      prev_end = e0;
      ent += w & 0xff;
    }
    if (!ok) set_error(J.ctr, kErrBadBlock, (uint32_t)b);
    J.blk_nent[b] = ok ? (uint32_t)ent : 0;
  }
}

// Input block checksums, for jobs that ask for them: the check ReadBlock
// makes when ReadOptions::verify_checksums is set (table/format.cc:86-95; the
// reference build has it switched off with `&& 0`, and LevelDB sets it for a
// compaction's inputs from Options::paranoid_checks, db/version_set.cc:1239):
// the fixed32 after the type byte must be Mask(crc32c(contents + type)).  One
// warp per data block; runs before the blocks are parsed, so that a damaged
// block reports the checksum rather than whatever its bytes break.
__global__ void __launch_bounds__(256) k_verify_blocks(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t tab[256];
  __shared__ uint32_t s_skip;
  if (threadIdx.x == 0) s_skip = (!J.verify_checksums || J.ctr->error) ? 1u : 0u;
  crc_table_init(tab);
  __syncthreads();
  if (s_skip) return;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  for (uint64_t b = (uint64_t)blockIdx.x * nw + warp; b < nblk; b += (uint64_t)gridDim.x * nw) {
    // the index parse checked that the block and its 5-byte trailer lie in the table
    const uint32_t size = J.blk_size[b];
    if (size == kPseudoBlock) continue;  // a decoded form: no block bytes to check
    const uint8_t* p = J.in + J.blk_off[b];
    const uint32_t crc = warp_block_crc(J, tab, p, size, p[size]);
    if (lane == 0 && crc != ld_le32(p + size + 1)) set_error(J.ctr, kErrChecksum, (uint32_t)b);
  }
}

// Entries of merge child r start at the first block of its first table: one
// thread per table, the first table of each run writes the run's start.
__global__ void k_run_bounds(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  const bool bad = J.ctr->error != 0;  // the job fails; keep every read in bounds
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < J.n_tables;
       t += gridDim.x * blockDim.x) {
    const uint32_t run = J.tables[t].run;
    if (t == 0 || J.tables[t - 1].run != run)
      J.run_entry_begin_w[run] =
          bad ? 0 : J.blk_ent_base[min(J.tbl_block_base[t], J.cap_blocks_in)];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) J.run_entry_begin_w[J.n_runs] = J.ctr->n_entries_in;
}

// Decode of one block straight from global memory, one lane per restart run:
// the path for blocks that do not fit the shared-memory stage.
__device__ void decode_direct(const JobDev& J, uint64_t b, uint32_t lane) {
  BlockView v = block_view(J, b, J.in + J.blk_off[b]);
  uint64_t ent_carry = J.blk_ent_base[b];
  uint64_t key_carry;
  if (J.reserve_keys) {
    // single pass: check every run and sum the block's key bytes first, then
    // reserve them in the key arena
    uint64_t kb = 0;
    uint32_t maxk = 0;
    bool ok = v.ok, sk = false;
    for (uint32_t r = lane; ok && r < v.nr; r += 32) {
      uint64_t s, e, rk = 0;
      uint32_t cnt;
      run_bounds(v, r, &s, &e, &cnt);
      if (s > e || e > v.ra || !walk_run(v.p + s, v.p + e, cnt, &rk, &maxk, &sk)) ok = false;
      kb += rk;
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    const bool any_short = __any_sync(0xffffffffu, sk);
    kb = warp_sum(kb);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
    uint64_t base = 0;
    int fail = 0;
    if (lane == 0) {
      fail = 1;
      if (!all_ok) set_error(J.ctr, kErrBadBlock, (uint32_t)b);
      else if (any_short) set_error(J.ctr, kErrShortKey, (uint32_t)b);
      else if (maxk > J.max_key_len) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
      else {
        base = atomicAdd((unsigned long long*)&J.ctr->key_cursor, (unsigned long long)kb);
        if (base + kb > J.cap_key_bytes) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
        else fail = 0;
      }
      atomicMax(&J.ctr->max_klen, maxk);
    }
    if (__shfl_sync(0xffffffffu, fail, 0)) return;
    key_carry = __shfl_sync(0xffffffffu, base, 0);
  } else {
    key_carry = J.blk_key_base[b];
  }
  for (uint32_t r0 = 0; r0 < v.nr; r0 += 32) {
    const uint32_t r = r0 + lane;
    uint64_t s = 0, e = 0, rk = 0;
    uint32_t cnt = 0, maxk = 0;
    bool sk = false;
    if (r < v.nr) {
      run_bounds(v, r, &s, &e, &cnt);
      walk_run(v.p + s, v.p + e, cnt, &rk, &maxk, &sk);
    }
    uint64_t cnt_tot, kb_tot;
    uint64_t ent = warp_excl<uint64_t>(cnt, &cnt_tot) + ent_carry;
    uint64_t kpos = warp_excl<uint64_t>(rk, &kb_tot) + key_carry;
    ent_carry += cnt_tot;
    key_carry += kb_tot;
    if (r < v.nr) {
      const uint8_t* p = v.p + s;
      const uint8_t* lim = v.p + e;
      uint64_t prev = kpos;
      for (uint32_t k = 0; k < cnt; k++) {
        uint32_t sh, ns, vl;
        const uint8_t* q = entry_header(p, lim, &sh, &ns, &vl);
        if (!q) break;
        const uint32_t kl = sh + ns;
        if (kpos + kl > J.cap_key_bytes || ent >= J.cap_entries) {
          set_error(J.ctr, kErrArenaOverflow, (uint32_t)b);
          return;
        }
        uint8_t* dst = J.keys + kpos;
        for (uint32_t i = 0; i < sh; i++) dst[i] = J.keys[prev + i];
        for (uint32_t i = 0; i < ns; i++) dst[sh + i] = q[i];
        J.e_koff[ent] = (uint32_t)kpos;
        J.e_klen[ent] = kl;
        J.e_voff[ent] = (uint32_t)((q + ns) - J.in);
        J.e_vlen[ent] = vl;
        J.e_pfx[ent] = user_prefix(dst, kl);
        J.e_tag[ent] = ld_le64(dst + kl - 8);
        prev = kpos;
        kpos += kl;
        ent++;
        p = q + ns + vl;
      }
    }
  }
}

// Decode of one staged block.  Lanes first walk the restart runs (one lane
// per run, headers only) and record every entry's key-delta position, shared
// prefix and lengths; then, 32 entries at a time, the warp rebuilds the keys
// in entry order in shared memory (lanes over bytes: the shared prefix is the
// front of the previous key, already rebuilt), writes them out with 16-byte
// stores, and writes the descriptors one lane per entry.
__device__ bool decode_staged(const JobDev& J, uint64_t b, uint32_t lane, const uint8_t* st,
                              DecWarpSmem& W) {
  BlockView v = block_view(J, b, st);
  const uint32_t nent = J.blk_nent[b];
  if (nent > kDecMaxEnt) return false;
  // pass 1: headers of every entry, one lane per restart run; the checks of
  // the counting walk (bounds, no shared prefix at a restart, shared prefix
  // within the previous key, runs parsed exactly to their end, keys of at
  // least 8 bytes) are made here too
  uint32_t carry = 0;
  bool long_key = false, bad = !v.ok, short_key = false;
  uint64_t rk = 0;
  uint32_t maxk = 0;
  for (uint32_t r0 = 0; r0 < v.nr; r0 += 32) {
    const uint32_t r = r0 + lane;
    uint64_t s = 0, e = 0;
    uint32_t cnt = 0;
    if (r < v.nr) run_bounds(v, r, &s, &e, &cnt);
    uint32_t tot;
    const uint32_t e0 = warp_excl<uint32_t>(cnt, &tot) + carry;
    carry += tot;
    if (r < v.nr) {
      if (s > e || e > v.ra) bad = true;
      const uint8_t* p = st + s;
      const uint8_t* lim = st + (e > v.ra ? v.ra : e);
      uint32_t prev = 0;
      for (uint32_t k = 0; k < cnt && !bad; k++) {
        uint32_t sh, ns, vl;
        const uint8_t* q = entry_header(p, lim, &sh, &ns, &vl);
        if (!q || (k == 0 && sh != 0) || sh > prev) {
          bad = true;
          break;
        }
        const uint32_t kl = sh + ns;
        const uint32_t idx = e0 + k;
        if (idx < kDecMaxEnt) {
          W.dpos[idx] = (uint16_t)(q - st);
          W.sh[idx] = (uint16_t)sh;
          W.kl[idx] = (uint16_t)kl;
          W.vl[idx] = (uint16_t)vl;
        }
        if (kl > 0xffff) long_key = true;
        if (kl < 8) short_key = true;
        rk += kl;
        maxk = max(maxk, kl);
        prev = kl;
        p = q + ns + vl;
      }
      if (!bad && p != lim) bad = true;
    }
  }
  if (J.reserve_keys) {
    if (__any_sync(0xffffffffu, bad)) {
      if (lane == 0) set_error(J.ctr, kErrBadBlock, (uint32_t)b);
      return true;
    }
    if (__any_sync(0xffffffffu, short_key)) {
      if (lane == 0) set_error(J.ctr, kErrShortKey, (uint32_t)b);
      return true;
    }
  }
  if (__any_sync(0xffffffffu, long_key)) return false;
  __syncwarp();
  // pass 2: keys and descriptors, 32 entries at a time
  const uint64_t ebase = J.blk_ent_base[b];
  uint64_t kbase;
  if (J.reserve_keys) {
    // reserve this block's key bytes in the arena
    rk = warp_sum(rk);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
    uint64_t base = 0;
    bool retry = false;
    if (lane == 0) {
      atomicMax(&J.ctr->max_klen, maxk);
      if (maxk > J.max_key_len) {
        retry = true;
      } else {
        base = atomicAdd((unsigned long long*)&J.ctr->key_cursor, (unsigned long long)rk);
        retry = base + rk > J.cap_key_bytes;
      }
      if (retry) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
    }
    if (__shfl_sync(0xffffffffu, (int)retry, 0)) return true;
    kbase = __shfl_sync(0xffffffffu, base, 0);
  } else {
    kbase = J.blk_key_base[b];
  }
  const uint32_t voff0 = (uint32_t)J.blk_off[b];  // block offset in `in`
  for (uint32_t g0 = 0; g0 < nent; g0 += 32) {
    const uint32_t i = g0 + lane;
    const bool valid = i < nent;
    const uint32_t kl = valid ? W.kl[i] : 0;
    uint32_t gk;
    const uint32_t kofs = warp_excl<uint32_t>(kl, &gk);
    uint8_t* gdst = J.keys + kbase;
    const uint32_t kph = (uint32_t)(reinterpret_cast<uintptr_t>(gdst) & 15);
    // the rest of the block goes through the direct path (which rewrites
    // the whole block) when a group's keys overflow the buffers
    if (__any_sync(0xffffffffu, kl > kDecLastKey) || gk + kph + 16 > kDecKeyBuf) {
      // a single-pass block has reserved its key bytes already: a retry of
      // the whole job with counting keeps the layout simple
      if (J.reserve_keys) {
        if (lane == 0) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
        return true;
      }
      return false;
    }
    uint8_t* kb = W.keybuf + kph;
    const uint32_t cnt = min(32u, nent - g0);
    for (uint32_t e = 0; e < cnt; e++) {
      const uint32_t ie = g0 + e;
      const uint32_t esh = W.sh[ie], ekl = W.kl[ie], edp = W.dpos[ie];
      const uint32_t eofs = __shfl_sync(0xffffffffu, kofs, e);
      const uint32_t pofs = __shfl_sync(0xffffffffu, kofs, (e + 31) & 31);
      const uint8_t* prev = e == 0 ? W.lastkey : kb + pofs;
      uint8_t* d = kb + eofs;
      for (uint32_t t = lane; t < ekl; t += 32) d[t] = t < esh ? prev[t] : st[edp + t - esh];
      __syncwarp();
    }
    {
      // the group's last key is the next group's first prefix
      const uint32_t lofs = __shfl_sync(0xffffffffu, kofs, cnt - 1);
      const uint32_t lkl = W.kl[g0 + cnt - 1];
      for (uint32_t t = lane; t < lkl; t += 32) W.lastkey[t] = kb[lofs + t];
    }
    __syncwarp();
    // keys out: head bytes, 16-byte body, tail
    const uint32_t head = (16 - kph) & 15;
    const uint32_t h = head < gk ? head : gk;
    if (lane < h) gdst[lane] = kb[lane];
    const uint32_t body = (gk - h) & ~15u;
    const uint4* sv = reinterpret_cast<const uint4*>(kb + h);
    uint4* dv = reinterpret_cast<uint4*>(gdst + h);
    for (uint32_t c = lane; c < body / 16; c += 32) dv[c] = sv[c];
    const uint32_t t0 = h + body;
    if (t0 + lane < gk) gdst[t0 + lane] = kb[t0 + lane];
    if (valid) {
      const uint64_t e = ebase + i;
      const uint32_t ko = (uint32_t)(kbase + kofs);
      J.e_koff[e] = ko;
      J.e_klen[e] = kl;
      J.e_voff[e] = voff0 + W.dpos[i] + (kl - W.sh[i]);
      J.e_vlen[e] = W.vl[i];
      J.e_pfx[e] = user_prefix(kb + kofs, kl);
      J.e_tag[e] = ld_le64(kb + kofs + kl - 8);
    }
    kbase += gk;
    __syncwarp();
  }
  return true;
}

// One block (warp per block): a decoded-run pseudo block, or a staged block,
// or, when it does not fit the stage, the direct path.
__device__ __forceinline__ void decode_one(const JobDev& J, uint64_t b, uint32_t lane,
                                           DecWarpSmem& W) {
  if (J.blk_size[b] == kPseudoBlock) {
    uint64_t kb;
    uint32_t mk;
    if (!__all_sync(0xffffffffu, pseudo_entries(J, b, J.blk_ent_base[b], lane, 32, &kb, &mk))) {
      if (lane == 0) set_error(J.ctr, kErrBadEntry, (uint32_t)b);
      return;
    }
    uint64_t kbase = 0;
    if (J.reserve_keys) {
      // single pass: reserve the block's key bytes in the arena
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mk = max(mk, __shfl_xor_sync(0xffffffffu, mk, o));
      int retry = 0;
      if (lane == 0) {
        atomicMax(&J.ctr->max_klen, mk);
        if (mk > J.max_key_len) {
          retry = 1;
        } else {
          kbase = atomicAdd((unsigned long long*)&J.ctr->key_cursor, (unsigned long long)kb);
          retry = kbase + kb > J.cap_key_bytes;
        }
        if (retry) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
      }
      if (__shfl_sync(0xffffffffu, retry, 0)) return;
      kbase = __shfl_sync(0xffffffffu, kbase, 0);
    } else {
      kbase = J.blk_key_base[b];
    }
    pseudo_keys(J, b, J.blk_ent_base[b], kbase, lane);
    return;
  }
  const uint8_t* st = stage_block(J, b, W.stage, lane);
  if (!st || !decode_staged(J, b, lane, st, W)) decode_direct(J, b, lane);
  __syncwarp();
}

// Sparse blocks: few entries with long values (the job's blocks average at
// most kSparseEnt entries, the block at most 64 KiB).  Staging them would
// move every value byte for a few header and key bytes, so a warp takes
// kSparseGroup consecutive blocks: each lane walks its block's restart runs
// straight from global memory (headers only), recording every entry in the
// warp's arrays; one atomic reserves all their key spans; then the warp
// rebuilds each block's keys (shared prefix from the previous key, delta
// from global memory) and writes keys and descriptors.  Blocks that are not
// sparse in such a group go through decode_one.
constexpr uint32_t kSparseEnt = 8;
constexpr uint32_t kSparseGroup = 32;

__device__ __forceinline__ bool sparse_block(const JobDev& J, uint64_t b) {
  const uint32_t size = J.blk_size[b], nent = J.blk_nent[b];
  return size != kPseudoBlock && size <= 0xffff && nent > 0 && nent <= kSparseEnt &&
         size >= 128u * nent;
}

__device__ void decode_sparse_group(const JobDev& J, uint64_t g0, uint64_t nblk, uint32_t lane,
                                    DecWarpSmem& W) {
  const uint64_t b = g0 + lane;
  const bool mine = b < nblk && sparse_block(J, b);
  const unsigned mask = __ballot_sync(0xffffffffu, mine);
  // 1. one lane per sparse block: headers from global memory
  bool bad = false, short_key = false;
  uint32_t kb = 0, maxk = 0, nent = 0;
  if (mine) {
    const uint8_t* p = J.in + J.blk_off[b];
    const uint32_t size = J.blk_size[b];
    const uint32_t nr = ld_le32(p + size - 4);  // checked by k_block_restarts
    const uint32_t ra = size - 4 - 4 * nr;
    nent = J.blk_nent[b];
    uint32_t e = 0;
    for (uint32_t r = 0; r < nr && !bad; r++) {
      const uint32_t w = ld_le32(p + ra + 4 * r);
      const uint32_t cnt = w & 0xff;
      const uint8_t* q = p + (w >> 8);
      const uint8_t* lim = p + ((r + 1 < nr) ? (ld_le32(p + ra + 4 * (r + 1)) >> 8) : ra);
      uint32_t prev = 0;
      for (uint32_t k = 0; k < cnt; k++) {
        uint32_t sh, ns, vl;
        const uint8_t* d = entry_header(q, lim, &sh, &ns, &vl);
        if (!d || (k == 0 && sh != 0) || sh > prev || e >= nent) {
          bad = true;
          break;
        }
        const uint32_t kl = sh + ns;
        if (kl < 8) short_key = true;
        const uint32_t x = lane * kSparseEnt + e;
        W.dpos[x] = (uint16_t)(d - p);
        W.sh[x] = (uint16_t)sh;
        W.kl[x] = (uint16_t)kl;
        W.vl[x] = (uint16_t)vl;
        kb += kl;
        maxk = max(maxk, kl);
        prev = kl;
        q = d + ns + vl;
        e++;
      }
      if (!bad && q != lim) bad = true;
    }
    if (!bad && e != nent) bad = true;
    if (bad) set_error(J.ctr, kErrBadBlock, (uint32_t)b);
    else if (short_key) set_error(J.ctr, kErrShortKey, (uint32_t)b);
    else if (J.reserve_keys && maxk > J.max_key_len) set_error(J.ctr, kErrRetryExact, (uint32_t)b);
    atomicMax(&J.ctr->max_klen, maxk);
  }
  // 2. key spans: one reservation for the group (single pass), else the scan's
  const bool ok = mine && !bad && !short_key && (!J.reserve_keys || maxk <= J.max_key_len);
  const uint32_t need = ok ? kb : 0;
  uint64_t kbase = 0;
  if (J.reserve_keys) {
    uint32_t tot;
    const uint32_t ex = warp_excl<uint32_t>(need, &tot);
    uint64_t base = 0;
    if (lane == 0 && tot)
      base = atomicAdd((unsigned long long*)&J.ctr->key_cursor, (unsigned long long)tot);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (tot && base + tot > J.cap_key_bytes) {
      if (lane == 0) set_error(J.ctr, kErrRetryExact, (uint32_t)g0);
      return;
    }
    kbase = base + ex;
  } else if (mine) {
    kbase = J.blk_key_base[b];
  }
  __syncwarp();
  // 3. keys rebuilt in entry order and descriptors: one lane per block when
  // every key of the group fits a lane's 128-byte slice of the key buffer
  // (slices 132 bytes apart, so that the lanes' byte stores hit distinct
  // banks), else one block at a time across the warp
  const unsigned done = __ballot_sync(0xffffffffu, ok);
  uint32_t gmaxk = maxk;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gmaxk = max(gmaxk, __shfl_xor_sync(0xffffffffu, gmaxk, o));
  if (gmaxk <= 128) {
    if (ok) {
      const uint8_t* p = J.in + J.blk_off[b];
      const uint32_t voff0 = (uint32_t)J.blk_off[b];
      const uint64_t ebase = J.blk_ent_base[b];
      uint8_t* slice = W.keybuf + lane * 132;
      uint8_t* gdst = J.keys + kbase;
      uint32_t kofs = 0;
      for (uint32_t x = 0; x < nent; x++) {
        const uint32_t i = lane * kSparseEnt + x;
        const uint32_t esh = W.sh[i], ekl = W.kl[i], edp = W.dpos[i];
        for (uint32_t t = esh; t < ekl; t += 32)
          copy_small(slice + t, p + edp + (t - esh), min(32u, ekl - t));
        for (uint32_t t = 0; t < ekl; t++) gdst[kofs + t] = slice[t];
        const uint64_t e = ebase + x;
        J.e_koff[e] = (uint32_t)(kbase + kofs);
        J.e_klen[e] = ekl;
        J.e_voff[e] = voff0 + edp + (ekl - esh);
        J.e_vlen[e] = W.vl[i];
        J.e_pfx[e] = user_prefix(slice, ekl);
        J.e_tag[e] = ld_le64(slice + ekl - 8);
        kofs += ekl;
      }
    }
    __syncwarp();
  } else
  for (unsigned m = done; m; m &= m - 1) {
    const uint32_t L = __ffs(m) - 1;
    const uint64_t bb = g0 + L;
    const uint32_t n = __shfl_sync(0xffffffffu, nent, L);
    const uint64_t kb0 = __shfl_sync(0xffffffffu, kbase, L);
    const uint8_t* p = J.in + J.blk_off[bb];
    const uint32_t voff0 = (uint32_t)J.blk_off[bb];
    const uint64_t ebase = J.blk_ent_base[bb];
    uint8_t* kbuf = W.keybuf;  // at most kSparseEnt keys of at most 256 bytes (single pass)
    uint32_t kofs = 0, pofs = 0;
    const bool fits = __shfl_sync(0xffffffffu, kb, L) <= kDecKeyBuf;
    uint8_t* gdst = J.keys + kb0;
    for (uint32_t x = 0; x < n; x++) {
      const uint32_t i = L * kSparseEnt + x;
      const uint32_t esh = W.sh[i], ekl = W.kl[i], edp = W.dpos[i];
      if (fits) {
        uint8_t* d = kbuf + kofs;
        for (uint32_t t = lane; t < ekl; t += 32)
          d[t] = t < esh ? kbuf[pofs + t] : __ldg(p + edp + t - esh);
      } else {
        // longer keys (exact reruns): built in place in the arena, one key at a time
        uint8_t* d = gdst + kofs;
        for (uint32_t t = lane; t < ekl; t += 32) d[t] = t < esh ? gdst[pofs + t] : p[edp + t - esh];
      }
      __syncwarp();
      if (lane == 0) {
        const uint64_t e = ebase + x;
        J.e_koff[e] = (uint32_t)(kb0 + kofs);
        J.e_klen[e] = ekl;
        J.e_voff[e] = voff0 + edp + (ekl - esh);
        J.e_vlen[e] = W.vl[i];
      }
      pofs = kofs;
      kofs += ekl;
    }
    __syncwarp();
    if (fits) {
      for (uint32_t t = lane; t < kofs; t += 32) gdst[t] = kbuf[t];
    }
    // prefixes and tags, one lane per entry
    if (lane < n) {
      const uint32_t i = L * kSparseEnt + lane;
      uint32_t o = 0;
      for (uint32_t x = 0; x < lane; x++) o += W.kl[L * kSparseEnt + x];
      const uint8_t* k = fits ? kbuf + o : gdst + o;
      const uint32_t kl = W.kl[i];
      J.e_pfx[ebase + lane] = user_prefix(k, kl);
      J.e_tag[ebase + lane] = ld_le64(k + kl - 8);
    }
    __syncwarp();
  }
  // 4. the group's other blocks
  const unsigned rest = __ballot_sync(0xffffffffu, b < nblk && !mine);
  for (unsigned m = rest; m; m &= m - 1) decode_one(J, g0 + (__ffs(m) - 1), lane, W);
}

// Jobs whose blocks are not sparse: one warp per block.
__global__ void __launch_bounds__(kDecWarps * 32) k_block_decode(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  extern __shared__ __align__(16) uint8_t dec_smem[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  DecWarpSmem& W = reinterpret_cast<DecWarpSmem*>(dec_smem)[warp];
  if (J.ctr->error || J.sparse_blocks) return;
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  for (uint64_t b = (uint64_t)blockIdx.x * kDecWarps + warp; b < nblk;
       b += (uint64_t)gridDim.x * kDecWarps)
    decode_one(J, b, lane, W);
}

// Jobs whose blocks are sparse: one warp per group of kSparseGroup blocks
// (a separate kernel, so that its registers do not weigh on the dense path).
__global__ void __launch_bounds__(kDecWarps * 32) k_block_decode_sparse(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  extern __shared__ __align__(16) uint8_t dec_smem[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  DecWarpSmem& W = reinterpret_cast<DecWarpSmem*>(dec_smem)[warp];
  if (J.ctr->error || !J.sparse_blocks) return;
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  for (uint64_t g = (uint64_t)blockIdx.x * kDecWarps + warp; g * kSparseGroup < nblk;
       g += (uint64_t)gridDim.x * kDecWarps)
    decode_sparse_group(J, g * kSparseGroup, nblk, lane, W);
}

__global__ void k_entries_from_offsets(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  const uint64_t n = J.cap_entries;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t ko = J.src_koffs[i], kl = J.src_koffs[i + 1] - ko;
    if (kl < 8) {
      set_error(J.ctr, kErrShortKey, (uint32_t)i);
      continue;
    }
    J.e_koff[i] = (uint32_t)ko;
    J.e_klen[i] = (uint32_t)kl;
    J.e_voff[i] = (uint32_t)J.src_voffs[i];
    J.e_vlen[i] = (uint32_t)(J.src_voffs[i + 1] - J.src_voffs[i]);
    J.e_pfx[i] = user_prefix(J.keys + ko, (uint32_t)kl);
    J.e_tag[i] = ld_le64(J.keys + ko + kl - 8);
    J.k_koff[i] = (uint32_t)ko;
    J.k_klen[i] = (uint32_t)kl;
    J.k_voff[i] = (uint32_t)J.src_voffs[i];
    J.k_vlen[i] = (uint32_t)(J.src_voffs[i + 1] - J.src_voffs[i]);
  }
}

}  // namespace

void launch_table_index_count(const Batch& bt, cudaStream_t st) {
  note_launch(), k_table_index_count<<<dim3(bt.max_tables, bt.B), 1024, 0, st>>>(bt.d);
}
void launch_table_index_entries(const Batch& bt, cudaStream_t st) {
  note_launch(), k_table_index_entries<<<dim3(bt.max_tables, bt.B), 1024, 0, st>>>(bt.d);
}

static void dec_smem_attr(const void* fn) {
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(kDecWarps * sizeof(DecWarpSmem)));
}

static unsigned dec_ctas(const Batch& bt) {
  // grid-stride over the device-side block count: 3 CTAs per SM x 8 waves in
  // total, shared out among the jobs of the batch
  const uint64_t cap = std::max<uint64_t>(1, bt.ctas_per_job ? bt.ctas_per_job : 148 * 3 * 8 / bt.B);
  return grid_x(bt.max_blocks_in, kDecWarps, cap);
}

void decode_kernel_attributes() {
  dec_smem_attr((const void*)k_block_count);
  dec_smem_attr((const void*)k_block_decode);
  dec_smem_attr((const void*)k_block_decode_sparse);
}

void launch_block_count(const Batch& bt, cudaStream_t st) {
  note_launch(), k_block_count<<<dim3(dec_ctas(bt), bt.B), kDecWarps * 32,
                                 kDecWarps * sizeof(DecWarpSmem), st>>>(bt.d);
}
void launch_block_restarts(const Batch& bt, cudaStream_t st) {
  note_launch(), k_block_restarts<<<dim3(grid_x(bt.max_blocks_in, 256, 148 * 8), bt.B), 256, 0, st>>>(
      bt.d);
}
void launch_verify_blocks(const Batch& bt, cudaStream_t st) {
  if (!bt.any_verify) return;
  note_launch(), k_verify_blocks<<<dim3(grid_x(bt.max_blocks_in, 8, 148 * 8), bt.B), 256, 0, st>>>(
      bt.d);
}
void launch_run_bounds(const Batch& bt, cudaStream_t st) {
  note_launch(), k_run_bounds<<<dim3((bt.max_tables + 127) / 128 + 1, bt.B), 128, 0, st>>>(bt.d);
}
void launch_block_decode(const Batch& bt, cudaStream_t st) {
  note_launch(), k_block_decode<<<dim3(dec_ctas(bt), bt.B), kDecWarps * 32,
                                  kDecWarps * sizeof(DecWarpSmem), st>>>(bt.d);
  note_launch(), k_block_decode_sparse<<<dim3(dec_ctas(bt), bt.B), kDecWarps * 32,
                                         kDecWarps * sizeof(DecWarpSmem), st>>>(bt.d);
}
void launch_entries_from_offsets(const Batch& bt, cudaStream_t st) {
  note_launch(), k_entries_from_offsets<<<dim3(grid_x(bt.max_entries, 256, 148 * 8), bt.B), 256, 0,
                                          st>>>(bt.d);
}

}  // namespace lc
