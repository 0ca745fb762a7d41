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
    if (threadIdx.x == 0) {
      J.tbl_nblocks[t] = (uint32_t)((J.dec_runs[t].n + kDecRunBlock - 1) / kDecRunBlock);
      J.tbl_unit[t] = 0;
    }
    return;
  }
  const uint8_t* base = J.in + T.off;
  __shared__ uint64_t s_ioff, s_isize;
  __shared__ uint32_t s_nr, s_ok;
  __shared__ uint32_t s_part[32], s_other[32];
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
    if (threadIdx.x == 0) {
      J.tbl_nblocks[t] = 0;
      J.tbl_unit[t] = 0;
    }
    return;
  }
  const uint8_t* ra = base + s_ioff + s_isize - 4 - 4ull * s_nr;
  uint32_t sum = 0, other = 0;  // entries; restart runs of other than one entry
  for (uint32_t r = threadIdx.x; r < s_nr; r += blockDim.x) {
    const uint32_t c = ld_le32(ra + 4ull * r) & 0xff;
    sum += c;
    other += c != 1;
  }
  sum = warp_sum(sum);
  other = warp_sum(other);
  if ((threadIdx.x & 31) == 0) {
    s_part[threadIdx.x >> 5] = sum;
    s_other[threadIdx.x >> 5] = other;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0, o = 0;
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; w++) s += s_part[w], o += s_other[w];
    J.tbl_nblocks[t] = s;
    J.tbl_unit[t] = o == 0;
  }
}

// Data block handles from the index blocks.  An index block whose restart
// runs each hold one entry (the table builder writes index blocks with a
// restart interval of 1) is cut into kIdxSplit parts, one CTA each, every
// thread parsing its own entries; any other is parsed by one CTA, the
// entries' places from a block-wide scan of the run counts.
constexpr uint32_t kIdxSplit = 16;

__global__ void k_table_index_entries(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  const uint32_t t = blockIdx.x / kIdxSplit, part = blockIdx.x % kIdxSplit;
  if (t >= J.n_tables) return;
  const TableDesc T = J.tables[t];
  const bool unit = J.tbl_unit[t] != 0;
  if (part != 0 && (T.cached || !unit)) return;
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
  if (unit) {
    const uint32_t r0 = (uint32_t)((uint64_t)nr * part / kIdxSplit);
    const uint32_t r1 = (uint32_t)((uint64_t)nr * (part + 1) / kIdxSplit);
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const uint64_t start = ld_le32(ra + 4ull * r) >> 8;
      const uint64_t end = (r + 1 < nr) ? (ld_le32(ra + 4ull * (r + 1)) >> 8) : ra_off;
      bool ok = start <= end && end <= ra_off;
      const uint8_t* p = idx + start;
      const uint8_t* lim = idx + end;
      uint32_t sh, ns, vl;
      const uint8_t* q = ok ? entry_header(p, lim, &sh, &ns, &vl) : nullptr;
      uint64_t b_off = 0, b_size = 0;
      const uint8_t* h = nullptr;
      if (q) {
        q += ns;
        h = get_varint64(q, q + vl, &b_off);
        if (h) h = get_varint64(h, q + vl, &b_size);
      }
      const uint64_t o = out_base + r;
      ok = h && b_off <= T.size && b_size + kTrailer <= T.size - b_off && o < out_end &&
           o < J.cap_blocks_in && q + vl == lim;
      if (ok) {
        J.blk_off[o] = T.off + b_off;
        J.blk_size[o] = (uint32_t)b_size;
        J.blk_run[o] = T.run;
      } else {
        set_error(J.ctr, kErrBadIndex, t);
      }
    }
    return;
  }
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

// Per-warp shared memory of the counting walk (k_block_count), and the key
// buffers of the decode.
constexpr uint32_t kDecWarps = 4;
constexpr uint32_t kDecStage = 8448;    // data block bytes + 16-byte phase
constexpr uint32_t kDecKeyBuf = 4096 + 32;  // a round's keys + phase
constexpr uint32_t kDecLastKey = 256;   // longest key the decode's buffers carry
struct DecWarpSmem {
  uint8_t stage[kDecStage];
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

// ---------------------------------------------------------------------------
// Decode of the data blocks into the entry arrays, in two passes.
//
// Pass 1 (k_decode_walk): one warp per group of dec_group consecutive data
// blocks (32, or 8 for blocks of many entries).  The group's restart runs,
// one lane per run in rounds of 32, walk their entry headers straight from
// global memory (the lines a run's headers lie in are read once, through L1)
// with the checks of the counting walk, and write one 16-byte record per
// entry -- where its key delta lies, its shared and key lengths, its value's
// length and place -- and its key length.  A pseudo block (a decoded run,
// from the decoded form of an earlier output) is cut into runs of
// kDecRunSlice entries whose records come from that form.
//
// A scan of the key lengths gives every key its place in the arena (keys in
// entry order).
//
// Pass 2 (k_decode_keys): one warp per unit of about kDecUnit entries, cut
// at entries without a shared prefix (every restart has none), in rounds of
// 32, one lane per entry: each lane copies its key delta into the warp's key
// buffer at the key's place; the shared prefixes then follow in entry order
// (a key's prefix is the head of the previous key, complete by then); the
// round's keys go out to the arena with 16-byte stores and the entry arrays
// with coalesced stores.  The round's last key carries into the next round;
// a round whose keys do not fit the buffer is built in the arena directly.
constexpr uint32_t kDecGroupMax = 32;   // data blocks per warp in pass 1
constexpr uint32_t kDecRunSlice = 16;   // pseudo-block entries per lane
constexpr uint32_t kDecUnit = 256;      // entries per warp in pass 2
constexpr uint32_t kDecPseudo = 0xffffu;  // shared length of a pseudo entry's record

// Record of entry e: x key delta offset in `in` (a pseudo entry: its block),
// y shared length | key length << 16, z value length, w value offset in `in`.
__device__ __forceinline__ uint4 dec_record(uint32_t src, uint32_t sh, uint32_t kl, uint32_t vl,
                                            uint32_t voff) {
  return make_uint4(src, sh | (kl << 16), vl, voff);
}

__global__ void __launch_bounds__(256) k_decode_walk(const JobDev* __restrict__ jobs) {
  __shared__ JobDev s_job;
  copy_job(jobs + blockIdx.y, &s_job);
  __syncthreads();
  const JobDev& J = s_job;
  __shared__ uint32_t s_rb[8][kDecGroupMax + 1];  // per warp: first run of each block of its group
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (J.ctr->error) return;
  const uint64_t nblk = min(J.ctr->n_blocks_in, J.cap_blocks_in);
  const uint32_t G = J.dec_group;
  const uint64_t ngrp = (nblk + G - 1) / G;
  for (uint64_t g = (uint64_t)blockIdx.x * 8 + warp; g < ngrp; g += (uint64_t)gridDim.x * 8) {
    const uint64_t g0 = g * G;
    // runs of the lane's block (a pseudo block: slices of its entries)
    uint32_t nr = 0;
    if (lane < G && g0 + lane < nblk) {
      const uint64_t b = g0 + lane;
      const uint32_t size = J.blk_size[b];
      if (size == kPseudoBlock) {
        nr = (J.blk_nent[b] + kDecRunSlice - 1) / kDecRunSlice;
      } else {
        nr = ld_le32(J.in + J.blk_off[b] + size - 4);  // checked by k_block_restarts
      }
    }
    uint32_t nrt;
    s_rb[warp][lane] = warp_excl<uint32_t>(nr, &nrt);
    if (lane == 0) s_rb[warp][kDecGroupMax] = nrt;
    __syncwarp();
    uint64_t kb = 0;
    uint32_t maxk = 0;
    bool bad = false, short_key = false, long_key = false;
    for (uint32_t q0 = 0; q0 < nrt; q0 += 32) {
      const uint32_t q = q0 + lane;
      if (q >= nrt) continue;
      // the block of run q: the last with its first run at or before q
      uint32_t lo = 0, hi = G;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_rb[warp][mid] <= q) lo = mid;
        else hi = mid;
      }
      const uint64_t b = g0 + lo;
      const uint32_t r = q - s_rb[warp][lo];
      const uint64_t ebase = J.blk_ent_base[b];
      const uint32_t size = J.blk_size[b];
      if (size == kPseudoBlock) {
        uint32_t t;
        uint64_t j0, j1;
        const DecRun& R = pseudo_block(J, b, &t, &j0, &j1);
        const TableDesc& T = J.tables[t];
        const uint64_t ja = j0 + (uint64_t)r * kDecRunSlice, jz = min(j1, ja + kDecRunSlice);
        for (uint64_t j = ja; j < jz; j++) {
          const uint32_t kl = (uint32_t)(R.kcum[j + 1] - R.kcum[j]);
          const uint32_t vl = R.vlen[j], vp = R.vpos[j];
          if (kl < 8) short_key = true;
          if (kl > 0xffff) long_key = true;
          if ((uint64_t)vp + vl > T.size) bad = true;
          const uint64_t e = ebase + (j - j0);
          J.e_rec[e] = dec_record((uint32_t)b, kDecPseudo, kl, vl, (uint32_t)(T.off + vp));
          J.e_klen[e] = kl;
          kb += kl;
          maxk = max(maxk, kl);
        }
        continue;
      }
      const uint8_t* p = J.in + J.blk_off[b];
      const uint32_t nrb = ld_le32(p + size - 4);
      const uint32_t ra = size - 4 - 4 * nrb;
      const uint32_t w = ld_le32(p + ra + 4 * r);
      const uint32_t cnt = w & 0xff;
      const uint32_t s = w >> 8, e = (r + 1 < nrb) ? (ld_le32(p + ra + 4 * (r + 1)) >> 8) : ra;
      uint32_t before = 0;  // entries of the block's earlier runs
      for (uint32_t x = 0; x < r; x++) before += ld_le32(p + ra + 4 * x) & 0xff;
      const uint8_t* qp = p + s;
      const uint8_t* lim = p + e;  // run ranges checked by k_block_restarts
      const uint32_t boff = (uint32_t)J.blk_off[b];
      // the record arrays in registers: the stores below cannot then make the
      // compiler reload them from the job descriptor
      uint4* const rec = J.e_rec + ebase + before;
      uint32_t* const klen = J.e_klen + ebase + before;
      uint32_t prev = 0;
      for (uint32_t k = 0; k < cnt; k++) {
        uint32_t sh, ns, vl;
        const uint8_t* d = entry_header(qp, lim, &sh, &ns, &vl);
        if (!d || (k == 0 && sh != 0) || sh > prev) {
          bad = true;
          break;
        }
        const uint32_t kl = sh + ns;
        if (kl < 8) short_key = true;
        if (kl > 0xffff || sh >= kDecPseudo) long_key = true;
        const uint32_t doff = boff + (uint32_t)(d - p);
        rec[k] = dec_record(doff, sh, kl, vl, doff + ns);
        klen[k] = kl;
        kb += kl;
        maxk = max(maxk, kl);
        prev = kl;
        qp = d + ns + vl;
      }
      if (!bad && qp != lim) bad = true;
    }
    const bool any_bad = __any_sync(0xffffffffu, bad);
    const bool any_short = __any_sync(0xffffffffu, short_key);
    const bool any_long = __any_sync(0xffffffffu, long_key);
    kb = warp_sum(kb);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
    if (lane == 0) {
      atomicMax(&J.ctr->max_klen, maxk);
      atomicAdd((unsigned long long*)&J.ctr->key_total, (unsigned long long)kb);
      if (any_bad) set_error(J.ctr, kErrBadBlock, (uint32_t)g0);
      else if (any_short) set_error(J.ctr, kErrShortKey, (uint32_t)g0);
      else if (any_long) set_error(J.ctr, kErrLimit, 4);
      else if (J.reserve_keys && maxk > J.max_key_len) set_error(J.ctr, kErrRetryExact, (uint32_t)g0);
    }
    __syncwarp();
  }
}

// The arena holds every key (k_decode_keys checks it before writing any).
__global__ void k_decode_fit(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (threadIdx.x == 0 && !J.ctr->error && J.ctr->key_total > J.cap_key_bytes)
    set_error(J.ctr, J.reserve_keys ? kErrRetryExact : kErrArenaOverflow, 5);
}

struct DecKeysSmem {
  uint8_t buf[kDecKeyBuf];    // the round's keys, at the arena's 16-byte phase
  uint8_t last[kDecLastKey];  // the previous round's last key
};

// The key bytes a record points at: the key delta in `in`, or a pseudo
// entry's whole key in its decoded run.
__device__ __forceinline__ const uint8_t* dec_delta(const JobDev& J, uint64_t e, uint4 rec) {
  if ((rec.y & 0xffff) == kDecPseudo) {
    uint32_t t;
    uint64_t j0, j1;
    const uint64_t b = rec.x;
    const DecRun& R = pseudo_block(J, b, &t, &j0, &j1);
    return R.keys + R.kcum[j0 + (e - J.blk_ent_base[b])];
  }
  return J.in + rec.x;
}

// First entry at or after e (below n) without a shared prefix, else n.
__device__ __forceinline__ uint64_t dec_unit_start(const JobDev& J, uint64_t e, uint64_t n,
                                                   uint32_t lane) {
  for (; e < n; e += 32) {
    const uint64_t x = e + lane;
    const uint32_t sh = x < n ? (J.e_rec[x].y & 0xffff) : 1u;
    const unsigned m = __ballot_sync(0xffffffffu, x < n && (sh == 0 || sh == kDecPseudo));
    if (m) return e + (__ffs(m) - 1);
  }
  return n;
}

__global__ void __launch_bounds__(256) k_decode_keys(const JobDev* __restrict__ jobs) {
  __shared__ JobDev s_job;
  copy_job(jobs + blockIdx.y, &s_job);
  __syncthreads();
  const JobDev& J = s_job;
  __shared__ __align__(16) DecKeysSmem s_w[8];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  DecKeysSmem& W = s_w[warp];
  if (J.ctr->error) return;
  const uint64_t n = J.ctr->n_entries_in;
  const uint64_t nunits = (n + kDecUnit - 1) / kDecUnit;
  for (uint64_t u = (uint64_t)blockIdx.x * 8 + warp; u < nunits; u += (uint64_t)gridDim.x * 8) {
    const uint64_t e0 = u == 0 ? 0 : dec_unit_start(J, u * kDecUnit, n, lane);
    const uint64_t e1 = dec_unit_start(J, (u + 1) * kDecUnit, n, lane);
    bool last_staged = true;  // the previous key is in W.last (not needed at a unit start)
    uint64_t last_at = 0;     // else its arena offset
    for (uint64_t r0 = e0; r0 < e1; r0 += 32) {
      const uint64_t e = r0 + lane;
      const bool valid = e < e1;
      const uint32_t cnt = (uint32_t)min(32ull, (unsigned long long)(e1 - r0));
      const uint4 rec = valid ? J.e_rec[e] : make_uint4(0, 0, 0, 0);
      const uint32_t kl = rec.y >> 16;
      const uint32_t sh = (rec.y & 0xffff) == kDecPseudo ? 0 : (rec.y & 0xffff);
      const uint8_t* src = valid ? dec_delta(J, e, rec) : nullptr;
      const uint64_t kpos = J.e_koff[r0];  // arena offset of the round's first key
      uint32_t tot;
      const uint32_t ko = warp_excl<uint32_t>(kl, &tot);  // offset within the round
      uint32_t mk = kl;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mk = max(mk, __shfl_xor_sync(0xffffffffu, mk, o));
      uint8_t* gdst = J.keys + kpos;
      const uint32_t kph = (uint32_t)(reinterpret_cast<uintptr_t>(gdst) & 15);
      const uint32_t sh0 = __shfl_sync(0xffffffffu, sh, 0);
      const uint32_t lkl = __shfl_sync(0xffffffffu, kl, cnt - 1);
      const uint32_t lko = __shfl_sync(0xffffffffu, ko, cnt - 1);
      if (tot + kph + 16 <= kDecKeyBuf && mk <= kDecLastKey && (sh0 == 0 || last_staged)) {
        uint8_t* kb = W.buf + kph;
        // deltas, every lane at once
        if (valid) {
          const uint32_t dl = kl - sh;
          for (uint32_t t = 0; t < dl; t += 32) copy_small_w(kb + ko + sh + t, src + t, min(32u, dl - t));
        }
        __syncwarp();
        // shared prefixes.  Within the round, an entry z without a shared
        // prefix holds its whole key as its delta; for the entries after it
        // (up to the next such entry), the bytes below the least shared
        // length since z are z's bytes -- every entry in between shares them.
        // Before the round's first such entry the same holds with the
        // previous round's last key.  Each other prefix byte is the own
        // (delta) byte of the nearest earlier entry whose shared length lies
        // below it (the entries in between share it), found by a walk back
        // that ends at the entry with that least shared length.
        const unsigned zmask = __ballot_sync(0xffffffffu, valid && sh == 0);
        const unsigned zbelow = zmask & (0xffffffffu >> (31 - lane));
        const int z = zbelow ? 31 - __clz(zbelow) : -1;
        const uint32_t koz = __shfl_sync(0xffffffffu, ko, z < 0 ? 0 : z);
        // segmented running minimum of the shared lengths since z (z excluded)
        uint32_t m = (valid && sh != 0) ? sh : 0xffffffffu;
        bool seg = valid && sh == 0;  // this lane's range reaches a segment head
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, m, o);
          const bool ys = __shfl_up_sync(0xffffffffu, seg, o);
          if (lane >= o && !seg) {
            m = min(m, y);
            seg = ys;
          }
        }
        if (!valid || sh == 0) m = 0;
        if (valid && m) {
          const uint8_t* from = z >= 0 ? kb + koz : W.last;
          for (uint32_t t = 0; t < m; t++) kb[ko + t] = from[t];
        }
        uint32_t lim = valid ? sh : 0;
        for (uint32_t d = 1; d < 32 && __any_sync(0xffffffffu, lim > m); d++) {
          const uint32_t j = lane >= d ? lane - d : lane;
          const uint32_t shj = __shfl_sync(0xffffffffu, sh, j);
          const uint32_t koj = __shfl_sync(0xffffffffu, ko, j);
          if (lim > m && lane >= d && shj < lim) {
            const uint32_t a = max(shj, m);
            for (uint32_t t = a; t < lim; t++) kb[ko + t] = kb[koj + t];
            lim = a;
          }
        }
        __syncwarp();
        // the round's last key for the next round; keys out: head bytes,
        // 16-byte body, tail bytes
        for (uint32_t t = lane; t < lkl; t += 32) W.last[t] = kb[lko + t];
        last_staged = true;
        const uint32_t head = (16 - kph) & 15;
        const uint32_t h = head < tot ? head : tot;
        if (lane < h) gdst[lane] = kb[lane];
        const uint32_t body = (tot - h) & ~15u;
        const uint4* sv = reinterpret_cast<const uint4*>(kb + h);
        uint4* dv = reinterpret_cast<uint4*>(gdst + h);
        for (uint32_t c = lane; c < body / 16; c += 32) dv[c] = sv[c];
        const uint32_t t0 = h + body;
        if (t0 + lane < tot) gdst[t0 + lane] = kb[t0 + lane];
        if (valid) {
          J.e_voff[e] = rec.w;
          J.e_vlen[e] = rec.z;
          J.e_pfx[e] = user_prefix(kb + ko, kl);
          J.e_tag[e] = ld_le64(kb + ko + kl - 8);
        }
      } else {
        // long keys: built in the arena, one key at a time, the lanes over
        // its bytes
        for (uint32_t i = 0; i < cnt; i++) {
          const uint32_t shi = __shfl_sync(0xffffffffu, sh, i);
          const uint32_t kli = __shfl_sync(0xffffffffu, kl, i);
          const uint32_t koi = __shfl_sync(0xffffffffu, ko, i);
          const uint32_t kpi = __shfl_sync(0xffffffffu, ko, (i + 31) & 31);
          const uint8_t* srci = reinterpret_cast<const uint8_t*>(__shfl_sync(
              0xffffffffu, (unsigned long long)reinterpret_cast<uintptr_t>(src), i));
          const uint8_t* prev = i ? gdst + kpi : (last_staged ? W.last : J.keys + last_at);
          uint8_t* d = gdst + koi;
          for (uint32_t t = lane; t < kli; t += 32) d[t] = t < shi ? prev[t] : srci[t - shi];
          __syncwarp();
        }
        last_at = kpos + lko;
        last_staged = lkl <= kDecLastKey;
        if (last_staged)
          for (uint32_t t = lane; t < lkl; t += 32) W.last[t] = gdst[lko + t];
        if (valid) {
          J.e_voff[e] = rec.w;
          J.e_vlen[e] = rec.z;
          J.e_pfx[e] = user_prefix(gdst + ko, kl);
          J.e_tag[e] = ld_le64(gdst + ko + kl - 8);
        }
      }
      __syncwarp();
    }
  }
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
  note_launch(), k_table_index_entries<<<dim3(bt.max_tables * kIdxSplit, bt.B), 1024, 0, st>>>(bt.d);
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

void decode_kernel_attributes() { dec_smem_attr((const void*)k_block_count); }

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
  // pass 1: one warp per group of 8 or 32 blocks; pass 2: one warp per unit
  // of kDecUnit entries; 8 warps per CTA, at most 8 CTAs per SM over the batch
  const uint64_t cap = std::max<uint64_t>(1, bt.ctas_per_job ? bt.ctas_per_job : 148 * 8 / bt.B);
  const uint64_t walk = (bt.max_blocks_in + 63) / 64, keys = (bt.max_entries + 8 * kDecUnit - 1) / (8 * kDecUnit);
  note_launch(), k_decode_walk<<<dim3((unsigned)std::max<uint64_t>(1, std::min(walk, cap)), bt.B), 256, 0,
                                 st>>>(bt.d);
  scan_batch(kScanDecKlen, bt, bt.max_entries, st);
  note_launch(), k_decode_fit<<<dim3(1, bt.B), 32, 0, st>>>(bt.d);
  note_launch(), k_decode_keys<<<dim3((unsigned)std::max<uint64_t>(1, std::min(keys, cap)), bt.B), 256, 0,
                                 st>>>(bt.d);
}
void launch_entries_from_offsets(const Batch& bt, cudaStream_t st) {
  note_launch(), k_entries_from_offsets<<<dim3(grid_x(bt.max_entries, 256, 148 * 8), bt.B), 256, 0,
                                          st>>>(bt.d);
}

}  // namespace lc
