// Encode: survivors -> output tables, byte-identical to the reference's
// TableBuilder driven by DoCompactionWork.
//
// Reference behaviour reproduced here:
// * BlockBuilder (table/block_builder.cc:56-114): prefix compression against
//   the previous key of the block, a restart every `restart_interval` entries,
//   LUDA restart words (offset << 8) | run length, size estimate
//   buffer + 4 * restarts + 4.
// * TableBuilder::Add / Flush (table/table_builder.cc:94-140): a block is
//   flushed as soon as the estimate reaches block_size after an add.
// * DoCompactionWork's output split (db/db_impl.cc:1105-1111, 1174-1180): a
//   file ends once its flushed bytes (blocks + 5-byte trailers) reach
//   max_file_size, or before the first survivor at or after a grandparent cut.
// * Index block (table_builder.cc:101-108, 228-234): restart interval 1, one
//   entry per block keyed by FindShortestSeparator / FindShortSuccessor
//   (db/dbformat.cc:69-101, util/comparator.cc:29-64).
// * Filter block (table/filter_block.cc:21-76, util/bloom.cc:28-54): one
//   bloom filter per 2 KiB of data-block start offsets over the user keys of
//   the blocks that start there; empty filters for skipped indices.
// * Metaindex, footer (table_builder.cc:213-252, table/format.cc:31-40) and
//   masked CRC32C trailers (table_builder.cc:178-195).
//
// Block boundaries form a chain: where the next block starts depends on where
// this one started (restart positions and the prefix-compression reset).  Each
// survivor s gets next(s), the start of the following block if a block began
// at s.  The chain from survivor 0 is resolved in three steps: per chunk of
// survivors, a table of exits for every possible entry point (pointer chasing
// in shared memory); one thread composing the tables across chunks; and a
// per-chunk chase from the resolved entry point that marks block starts.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "lc_device.cuh"
#include "lc_kernels.h"

namespace lc {

namespace {

constexpr uint32_t kNoSep = 0xffffffffu;
__constant__ char kFilterName[] = "filter.leveldb.BuiltinBloomFilter2";
constexpr uint32_t kFilterNameLen = 34;

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

__device__ __forceinline__ uint32_t bloom_bytes(uint64_t n, int bpk) {
  uint64_t bits = n * (uint64_t)bpk;
  if (bits < 64) bits = 64;
  return (uint32_t)((bits + 7) / 8);
}

__device__ __forceinline__ const uint8_t* kept_key(const JobDev& J, uint64_t k, uint32_t* len) {
  *len = J.k_klen[k];
  return J.keys + J.k_koff[k];
}

// Entry sizes as a restart entry (k_a) and as a prefix-compressed entry
// (k_b), the shared prefix with the previous survivor, survivor byte totals;
// also clears the block-start flags (n + 1 of them) for the chain.
__global__ void k_sizes(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_kept;
  unsigned long long kb = 0, vb = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) J.k_bstart[n] = 0;
  for (uint64_t k0 = (uint64_t)blockIdx.x * blockDim.x; k0 < n; k0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = k0 + threadIdx.x;
    if (k >= n) continue;
    J.k_bstart[k] = 0;
    uint32_t kl;
    const uint8_t* key = kept_key(J, k, &kl);
    const uint32_t vl = J.k_vlen[k];
    uint32_t shared = 0;
    if (k > 0) {
      uint32_t pl;
      const uint8_t* pk = kept_key(J, k - 1, &pl);
      const uint32_t m = min(kl, pl);
      while (shared < m && pk[shared] == key[shared]) shared++;
    }
    J.k_a[k] = 1 + varint_len(kl) + varint_len(vl) + kl + vl;
    J.k_b[k] = varint_len(shared) + varint_len(kl - shared) + varint_len(vl) + (kl - shared) + vl;
    J.k_shared[k] = shared;
    kb += kl;
    vb += vl;
  }
  // survivor byte totals, one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    kb += __shfl_xor_sync(0xffffffffu, kb, o);
    vb += __shfl_xor_sync(0xffffffffu, vb, o);
  }
  if ((threadIdx.x & 31) == 0 && (kb | vb)) {
    atomicAdd((unsigned long long*)&J.ctr->kept_key_bytes, kb);
    atomicAdd((unsigned long long*)&J.ctr->kept_value_bytes, vb);
  }
}

// TableBuilder's size estimate of a block [s, e] (buffer + 4 per restart +
// 4): the prefix-compressed sizes (k_pb, a prefix sum of k_b) plus, at every
// restart s + mR, the difference between the entry's restart size and its
// compressed size, plus the restart words.  `D` is that difference summed
// over the restarts up to segment m (the segment holding e).
__device__ __forceinline__ uint64_t block_est(const JobDev& J, uint64_t s, uint64_t e, uint64_t D,
                                              uint64_t m) {
  return J.k_pb[e + 1] - J.k_pb[s] + D + 4 * (m + 1) + 4;
}

// next(s): the first survivor of the block after the one that starts at s.
// The block ends after the first e whose estimate reaches block_size
// (TableBuilder::Add, table/table_builder.cc:120-123), or before the first
// grandparent cut after s, or at the end.  Restart segments (R survivors)
// are stepped through, then the segment that reaches block_size is binary
// searched: O(block / R + log R) loads instead of a walk over the block.
__device__ __forceinline__ uint64_t next_of(const JobDev& J, uint64_t s, uint64_t n) {
  const uint32_t R = J.restart_interval;
  const uint64_t bs = J.block_size;
  uint32_t lo = 0, hi = J.ctr->n_triggers;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (J.t_kept[mid] <= s) lo = mid + 1;
    else hi = mid;
  }
  const uint64_t limit = lo < J.ctr->n_triggers ? min(n, (uint64_t)J.t_kept[lo]) : n;
  uint64_t D = 0;
  for (uint64_t m = 0;; m++) {
    const uint64_t a = s + m * R;
    if (a >= limit) return limit;
    D += J.k_a[a] - J.k_b[a];
    const uint64_t z = min(a + R, limit);  // segment [a, z)
    if (block_est(J, s, z - 1, D, m) >= bs) {
      uint64_t l = a, h = z - 1;
      while (l < h) {
        const uint64_t mid = (l + h) >> 1;
        if (block_est(J, s, mid, D, m) >= bs) h = mid;
        else l = mid + 1;
      }
      return l + 1;
    }
  }
}

__global__ void k_next(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_kept;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t s0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t w0 = s0 - (threadIdx.x & 31);
  const uint64_t trips = n > w0 ? (n - w0 + stride - 1) / stride : 0;
  uint32_t jump = 0;
  for (uint64_t it = 0, s = s0; it < trips; it++, s += stride) {
    if (s < n) {
      const uint64_t nxt = next_of(J, s, n);
      J.k_next[s] = (uint32_t)nxt;
      jump = max(jump, (uint32_t)(nxt - s));
    }
  }
  // the longest block, one atomic per warp
  jump = __reduce_max_sync(0xffffffffu, jump);
  if ((threadIdx.x & 31) == 0 && jump) atomicMax(&J.ctr->max_jump, jump);
}


// Per chunk: exits of the chain for every entry point in the first `window`
// survivors of the chunk.  The chunk's next() values are staged in shared
// memory and cut into sub-chunks of kChainSub survivors: every (sub-chunk,
// entry point) pair is walked in parallel to the sub-chunk's exit, and the
// chunk's exits are composed from the sub-chunk exits (C / kChainSub steps
// per entry point instead of a walk over the whole chunk).  Windows wider
// than a sub-chunk walk the chunk directly.
constexpr uint32_t kChainSub = 256;

// Exit of sub-chunk s of a staged chunk [c0, c1) for entry point e (an
// absolute survivor index inside the sub-chunk's first `W`).
__device__ __forceinline__ uint64_t chain_sub_walk(const uint32_t* s_next, uint64_t c0, uint64_t c1,
                                                   uint64_t e, uint64_t sub_end) {
  const uint64_t end = min(c1, sub_end);
  while (e < end) e = s_next[e - c0];
  return e;
}

__global__ void k_chain_tables(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  extern __shared__ uint32_t s_next[];  // chunk next() values, then sub-chunk exits
  const uint64_t n = J.ctr->n_kept;
  const uint32_t C = J.chunk;
  const uint32_t W = J.ctr->max_jump;
  if (W > C) return;  // resolved sequentially instead
  const bool sub = W <= kChainSub;
  uint32_t* s_sub = s_next + C;  // (C / kChainSub) x W sub-chunk exits
  for (uint64_t c = blockIdx.x; c * C < n; c += gridDim.x) {
    const uint64_t c0 = c * C;
    const uint64_t c1 = min(n, c0 + C);
    __syncthreads();
    for (uint64_t i = threadIdx.x; i < c1 - c0; i += blockDim.x) s_next[i] = J.k_next[c0 + i];
    __syncthreads();
    if (!sub) {
      for (uint32_t i = threadIdx.x; i < W; i += blockDim.x) {
        uint64_t e = c0 + i;
        while (e < c1) e = s_next[e - c0];
        J.chunk_table[c * C + i] = (uint32_t)e;
      }
      continue;
    }
    const uint32_t nsub = (uint32_t)((c1 - c0 + kChainSub - 1) / kChainSub);
    for (uint32_t x = threadIdx.x; x < nsub * W; x += blockDim.x) {
      const uint32_t sb = x / W, i = x % W;
      const uint64_t s0 = c0 + (uint64_t)sb * kChainSub;
      s_sub[x] = (uint32_t)chain_sub_walk(s_next, c0, c1, s0 + i, s0 + kChainSub);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < W; i += blockDim.x) {
      uint64_t e = c0 + i;
      for (uint32_t sb = 0; sb < nsub && e < c1; sb++) {
        const uint64_t s0 = c0 + (uint64_t)sb * kChainSub;
        e = s_sub[sb * W + (uint32_t)(e - s0)];  // e lies in the sub-chunk's first W survivors
      }
      J.chunk_table[c * C + i] = (uint32_t)e;
    }
  }
}

// Exits of groups of kChainGroup chunks for every entry point in the first
// `window` survivors of the group's first chunk, by following the chunk
// tables (one thread per entry point).  Only when the chunk tables do not fit
// the resolving CTA's shared memory.
__global__ void k_chain_groups(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_kept;
  const uint32_t C = J.chunk;
  const uint32_t W = J.ctr->max_jump;
  if (W > C || n == 0) return;
  const uint64_t M = (n + C - 1) / C;
  if (M * W <= J.chain_smem_words) return;  // resolved from the chunk tables directly
  const uint64_t G = (M + kChainGroup - 1) / kChainGroup;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < G * W;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = x / W, i = x % W;
    const uint64_t c0 = g * kChainGroup, c1 = min(M, c0 + kChainGroup);
    uint64_t e = c0 * C + i;
    for (uint64_t c = c0; c < c1 && e < n; c++) e = J.chunk_table[c * C + (e - c * C)];
    J.group_table[g * C + i] = (uint32_t)e;
  }
}

// Entry point of every chunk: the chain from survivor 0 through the chunk
// tables.  Few chunks: one thread walks them over a shared-memory copy of the
// tables.  Many: one thread walks the group tables (in shared memory when they
// fit), then one thread per group walks its chunks from the group's entry
// point.
__global__ void k_chain_resolve(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  extern __shared__ uint32_t s_tab[];
  const uint64_t n = J.ctr->n_kept;
  const uint32_t C = J.chunk;
  const uint32_t W = J.ctr->max_jump;
  if (n == 0) return;
  if (W > C) {
    // blocks longer than a chunk: walk the whole chain
    if (threadIdx.x != 0) return;
    uint64_t e = 0;
    while (e < n) {
      J.k_bstart[e] = 1;
      e = J.k_next[e];
    }
    return;
  }
  const uint64_t M = (n + C - 1) / C;
  if (M * W <= J.chain_smem_words) {
    for (uint64_t i = threadIdx.x; i < M * W; i += blockDim.x)
      s_tab[i] = J.chunk_table[(i / W) * C + (i % W)];
    __syncthreads();
    if (threadIdx.x != 0) return;
    uint64_t e = 0;
    for (uint64_t c = 0; c < M; c++) {
      J.chunk_entry[c] = (uint32_t)e;
      if (e < n) e = s_tab[c * W + (e - c * C)];
    }
    return;
  }
  const uint64_t G = (M + kChainGroup - 1) / kChainGroup;
  const bool staged = G * W + G <= J.chain_smem_words;
  const bool entries_in_smem = G <= J.chain_smem_words;
  uint32_t* s_entry = s_tab + (staged ? G * W : 0);  // group entry points
  if (staged) {
    for (uint64_t i = threadIdx.x; i < G * W; i += blockDim.x)
      s_tab[i] = J.group_table[(i / W) * C + (i % W)];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t e = 0;
    for (uint64_t g = 0; g < G; g++) {
      const uint64_t c0 = g * kChainGroup;
      if (entries_in_smem) s_entry[g] = (uint32_t)e;
      else J.chunk_entry[c0] = (uint32_t)e;
      if (e < n)
        e = staged ? s_tab[g * W + (e - c0 * C)] : J.group_table[g * C + (e - c0 * C)];
    }
  }
  __syncthreads();
  for (uint64_t g = threadIdx.x; g < G; g += blockDim.x) {
    const uint64_t c0 = g * kChainGroup, c1 = min(M, c0 + kChainGroup);
    uint64_t e = entries_in_smem ? s_entry[g] : J.chunk_entry[c0];
    for (uint64_t c = c0; c < c1; c++) {
      J.chunk_entry[c] = (uint32_t)e;
      if (e < n) e = J.chunk_table[c * C + (e - c * C)];
    }
  }
}

// Block starts: each chunk's chain from its resolved entry point.  With
// sub-chunks, one thread finds the sub-chunks' entry points from their exits
// (recomputed as k_chain_tables does) and every sub-chunk is walked by its
// own thread.
__global__ void k_chain_mark(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  extern __shared__ uint32_t s_next[];
  const uint64_t n = J.ctr->n_kept;
  const uint32_t C = J.chunk;
  const uint32_t W = J.ctr->max_jump;
  if (W > C) return;
  const bool sub = W <= kChainSub;
  uint32_t* s_sub = s_next + C;
  uint32_t* s_entry = s_sub + (C / kChainSub) * (sub ? W : 0);  // sub-chunk entry points
  for (uint64_t c = blockIdx.x; c * C < n; c += gridDim.x) {
    const uint64_t c0 = c * C;
    const uint64_t c1 = min(n, c0 + C);
    __syncthreads();
    for (uint64_t i = threadIdx.x; i < c1 - c0; i += blockDim.x) s_next[i] = J.k_next[c0 + i];
    __syncthreads();
    if (!sub) {
      if (threadIdx.x == 0) {
        uint64_t e = J.chunk_entry[c];
        while (e < c1) {
          J.k_bstart[e] = 1;
          e = s_next[e - c0];
        }
      }
      continue;
    }
    const uint32_t nsub = (uint32_t)((c1 - c0 + kChainSub - 1) / kChainSub);
    for (uint32_t x = threadIdx.x; x < nsub * W; x += blockDim.x) {
      const uint32_t sb = x / W, i = x % W;
      const uint64_t s0 = c0 + (uint64_t)sb * kChainSub;
      s_sub[x] = (uint32_t)chain_sub_walk(s_next, c0, c1, s0 + i, s0 + kChainSub);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t e = J.chunk_entry[c];
      for (uint32_t sb = 0; sb < nsub; sb++) {
        s_entry[sb] = (uint32_t)e;
        const uint64_t s0 = c0 + (uint64_t)sb * kChainSub;
        if (e < c1) e = s_sub[sb * W + (uint32_t)(e - s0)];
      }
    }
    __syncthreads();
    for (uint32_t sb = threadIdx.x; sb < nsub; sb += blockDim.x) {
      const uint64_t s0 = c0 + (uint64_t)sb * kChainSub, send = min(c1, s0 + kChainSub);
      uint64_t e = s_entry[sb];
      while (e < send) {
        J.k_bstart[e] = 1;
        e = s_next[e - c0];
      }
    }
  }
}

// Output blocks: first survivor of each block, and the block's size (the
// block that starts at k ends where the chain says the next one starts).
__global__ void k_block_list(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_kept;
  const uint32_t R = J.restart_interval;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= n;
       k += (uint64_t)gridDim.x * blockDim.x) {
    if (k == n) {
      J.b_first[J.k_block[n]] = (uint32_t)n;
    } else if (J.k_bstart[k]) {
      const uint32_t b = J.k_block[k];
      J.b_first[b] = (uint32_t)k;
      const uint64_t e = J.k_next[k];
      uint64_t D = 0;
      for (uint64_t a = k; a < e; a += R) D += J.k_a[a] - J.k_b[a];
      const uint64_t nrest = (e - k + R - 1) / R;
      const uint32_t size = (uint32_t)(J.k_pb[e] - J.k_pb[k] + D + 4 * nrest + 4);
      J.b_size[b] = size;
      J.tmp32[b] = size + kTrailer;
    }
  }
}

// Like the block chain, a file's end depends on where it starts: every block
// b gets b_fnext[b], the first block of the next file if a file began at b (a
// binary search for the size cut, and the next forced block); one thread then
// walks the few file starts.

// t_blocks[i] = output block that starts at grandparent cut i (ascending).
__global__ void k_forced_blocks(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= J.ctr->n_triggers) return;
  const uint64_t kp = J.kept_pos[J.triggers[i]];
  J.t_blocks[i] = kp < J.ctr->n_kept ? J.k_block[kp] : (uint32_t)J.ctr->n_blocks_out;
}

__global__ void k_file_next(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t nb = J.ctr->n_blocks_out;
  const uint32_t nt = J.ctr->n_triggers;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x) {
    // first forced block after b
    uint32_t lo = 0, hi = nt;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (J.t_blocks[mid] <= b) lo = mid + 1;
      else hi = mid;
    }
    const uint64_t next_forced = lo < nt ? J.t_blocks[lo] : nb;
    // first block end where the file's flushed bytes reach max_file_size
    const uint64_t cum0 = J.b_cum[b];
    const uint64_t target =
        J.max_file_size > ~0ull - cum0 ? ~0ull : cum0 + J.max_file_size;  // saturating
    uint64_t sc;
    if (J.b_cum[nb] < target) {
      sc = nb - 1;
    } else {
      uint64_t l = b, h = nb - 1;
      while (l < h) {
        const uint64_t mid = (l + h) >> 1;
        if (J.b_cum[mid + 1] >= target) h = mid;
        else l = mid + 1;
      }
      sc = l;
    }
    J.b_fnext[b] = (uint32_t)(min(sc, next_forced - 1) + 1);
  }
}

// The file starts are the orbit of block 0 under b_fnext, which only moves
// forward: the CTA loads a tile of b_fnext at the walk's position into shared
// memory, one 16-byte load per thread from the 16-byte boundary at or below
// it, and thread 0 walks inside it; a step that leaves the tile reloads.
// (b_fnext has N >= n_blocks_out words and 16 bytes of padding, so the last
// vector load stays inside its allocation.)
constexpr uint32_t kFileTile = 4096;
constexpr uint32_t kFileThreads = kFileTile / 4;
__global__ void k_files(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  __shared__ __align__(16) uint32_t tile[kFileTile];
  __shared__ uint64_t s_b;
  __shared__ uint32_t s_f;
  __shared__ bool s_stop;
  const uint64_t nb = J.ctr->n_blocks_out;
  if (threadIdx.x == 0) {
    s_b = 0;
    s_f = 0;
    s_stop = nb == 0;
  }
  __syncthreads();
  while (!s_stop) {
    const uint64_t t0 = s_b & ~uint64_t(3);
    for (uint64_t i = threadIdx.x; 4 * i < kFileTile && t0 + 4 * i < nb; i += blockDim.x)
      reinterpret_cast<uint4*>(tile)[i] = reinterpret_cast<const uint4*>(J.b_fnext + t0)[i];
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t b = s_b;
      uint32_t f = s_f;
      while (b < nb && b < t0 + kFileTile) {
        const uint64_t end = tile[b - t0];
        if (f >= J.cap_files) {
          set_error(J.ctr, kErrLimit, 2);
          b = nb;
          break;
        }
        FileOut& F = J.files[f];  // first_kept / end_kept: k_block_layout
        F.first_block = (uint32_t)b;
        F.end_block = (uint32_t)end;
        f++;
        b = end;
      }
      s_b = b;
      s_f = f;
      s_stop = b >= nb;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) J.ctr->n_files = s_f;
}

__device__ __forceinline__ uint32_t file_of_block(const JobDev& J, uint64_t b) {
  uint32_t lo = 0, hi = J.ctr->n_files;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (J.files[mid].first_block <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ void block_layout_one(const JobDev& J, uint64_t b);

__global__ void k_block_layout(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t nb = J.ctr->n_blocks_out;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x)
    block_layout_one(J, b);
}

__device__ void block_layout_one(const JobDev& J, uint64_t b) {
  const uint32_t f = file_of_block(J, b);
  const uint32_t fb0 = J.files[f].first_block, fb1 = J.files[f].end_block;
  if (b == fb0) J.files[f].first_kept = J.b_first[b];
  if (b + 1 == fb1) J.files[f].end_kept = J.b_first[b + 1];
  const uint64_t base = J.b_cum[fb0];
  const uint64_t off = J.b_cum[b] - base;
  J.b_file[b] = f;
  J.b_off[b] = off;
  // filter group: blocks of this file whose start offsets share off >> 11
  uint32_t gbytes = 0, gkeys = 0;
  if (J.bits_per_key > 0) {
    const uint64_t j = off >> kFilterBaseLg;
    const bool start = (b == fb0) || (((J.b_cum[b - 1] - base) >> kFilterBaseLg) != j);
    if (start) {
      uint64_t n = 0;
      for (uint64_t bb = b; bb < fb1 && ((J.b_cum[bb] - base) >> kFilterBaseLg) == j; bb++)
        n += J.b_first[bb + 1] - J.b_first[bb];
      gkeys = (uint32_t)n;
      gbytes = bloom_bytes(n, J.bits_per_key) + 1;
    }
  }
  J.b_gbytes[b] = gbytes;
  J.b_gkeys[b] = gkeys;
  // index key for this block
  uint32_t llen;
  const uint8_t* lkey = kept_key(J, J.b_first[b + 1] - 1, &llen);
  const uint32_t ulen = llen - 8;
  uint32_t sep = kNoSep, ilen = llen;
  if (b + 1 < fb1) {
    uint32_t nlen;
    const uint8_t* nkey = kept_key(J, J.b_first[b + 1], &nlen);
    const uint32_t nul = nlen - 8;
    const uint32_t m = min(ulen, nul);
    uint32_t d = 0;
    while (d < m && lkey[d] == nkey[d]) d++;
    if (d < m) {
      const uint32_t db = lkey[d];
      if (db < 0xff && db + 1 < nkey[d] && d + 1 < ulen) {
        sep = d;
        ilen = d + 1 + 8;
      }
    }
  } else {
    uint32_t i = 0;
    while (i < ulen && lkey[i] == 0xff) i++;
    if (i < ulen && i + 1 < ulen) {
      sep = i;
      ilen = i + 1 + 8;
    }
  }
  const uint32_t hl = varint_len(off) + varint_len(J.b_size[b]);
  J.b_sep[b] = sep;
  J.b_ilen[b] = ilen;
  J.b_isize[b] = 1 + varint_len(ilen) + varint_len(hl) + ilen + hl;
}

__global__ void k_file_layout(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  const uint32_t nf = J.ctr->n_files;
  for (uint32_t f = threadIdx.x; f < nf; f += blockDim.x) {
    FileOut& F = J.files[f];
    const uint32_t fb0 = F.first_block, fb1 = F.end_block;
    const uint64_t D = J.b_cum[fb1] - J.b_cum[fb0];
    F.data_bytes = D;
    uint64_t meta_off;
    if (J.bits_per_key > 0) {
      const uint64_t o_last = J.b_cum[fb1 - 1] - J.b_cum[fb0];
      const uint32_t nfl = (uint32_t)((D >> kFilterBaseLg) +
                                      ((D >> kFilterBaseLg) == (o_last >> kFilterBaseLg) ? 1 : 0));
      const uint64_t Ft = J.b_gcum[fb1] - J.b_gcum[fb0];
      const uint64_t fsize = Ft + 4ull * nfl + 4 + 1;
      F.filter_off = D;
      F.filter_size = fsize;
      F.n_filters = nfl;
      meta_off = D + fsize + kTrailer;
      F.meta_size = 3 + kFilterNameLen + varint_len(D) + varint_len(fsize) + 8;
    } else {
      F.filter_off = 0;
      F.filter_size = 0;
      F.n_filters = 0;
      meta_off = D;
      F.meta_size = 8;
    }
    F.meta_off = meta_off;
    F.crc_acc[0] = F.crc_acc[1] = F.crc_acc[2] = 0;
    F.index_off = meta_off + F.meta_size + kTrailer;
    F.index_size = (J.b_icum[fb1] - J.b_icum[fb0]) + 4ull * (fb1 - fb0) + 4;
    F.size = F.index_off + F.index_size + kTrailer + kFooter;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t o = 0;
    for (uint32_t f = 0; f < nf; f++) {
      J.files[f].out_off = o;
      o += J.files[f].size;
    }
    J.ctr->bytes_out = o;
    // a single-pass job sized its output buffer from the input: rerun it
    // with exact counting instead of failing
    if (o > J.cap_out) set_error(J.ctr, J.reserve_keys ? kErrRetryExact : kErrLimit, 3);
  }
}

// One warp per output data block, assembled around the warp's shared-memory
// stage, which has the block's own 16-byte phase in global memory: stage
// position p is global byte dst - ph + p, ph = dst & 15.  Three steps:
//  1. Entries in rounds of 32, one lane per entry: entry sizes and output
//     offsets by a warp scan.  A key delta or value of at least kEncLong
//     bytes lists its whole 16-byte chunks in the warp's list of long
//     stretches (at most kEncMaxLong; a lane stages the chunks of a stretch
//     past the list itself).  Once the list is complete (the last round), the
//     listed chunks of the first two chunk rows are loaded, and while they
//     are in flight the lanes write entry headers, restart words, short
//     stretches whole and the unaligned heads and tails of long ones to the
//     stage.
//  2. The block's 16-byte chunks, lane l taking chunks l, l + 32, ..., each
//     loaded two chunks ahead of its use: a chunk inside a listed stretch is
//     read from global memory (five 4-byte loads and four funnel shifts at
//     any source alignment), any other from the stage.  A chunk wholly
//     inside the block and its type byte goes out with one 16-byte store,
//     and every chunk feeds the lane's share of the block CRC (crc_h5).  The
//     stage's first and last chunks are cleared before step 1, so the grid
//     bytes outside the message are zero and every chunk takes the same CRC
//     step; the initial all-ones register enters at the end, as its register
//     carried over the message's length (crc_ones).
//  3. The lanes' CRC shares combined, the trailer (type byte and CRC) into
//     the stage, and the partial chunks at both ends from the stage with byte
//     stores.
// A block that does not fit the stage takes the direct path.
constexpr uint32_t kEncWarps = 8;
constexpr uint32_t kEncStage = 6144;  // block + 5-byte trailer + 16-byte phase + read slack
constexpr uint32_t kEncLong = 33;     // stretches at least this long are read by chunks
constexpr uint32_t kEncMaxLong = 64;  // listed long stretches per block
constexpr uint32_t kEncFromInput = 0x80000000u;
struct EncWarp {
  uint32_t ls_c0[kEncMaxLong];   // first whole chunk (stage grid) | kEncFromInput
  uint32_t ls_n[kEncMaxLong];    // whole chunks
  uint32_t ls_src[kEncMaxLong];  // source offset of the first chunk (key arena or input)
  uint32_t ahead[5][32];         // next block: lane j's entry (key length, shared, value
                                 // length, key offset, value offset), copied ahead
  __align__(16) uint8_t stage[kEncStage];
};
constexpr size_t kEncSmem = (size_t)kEncWarps * sizeof(EncWarp);

// 16 bytes from src at any alignment: the five words holding them (the fifth
// only when src is not word aligned) and four funnel shifts.
__device__ __forceinline__ void load16(const uint8_t* src, uint32_t (&w)[4]) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = 8 * (uint32_t)(a & 3);
  uint32_t x[5];
#pragma unroll
  for (int i = 0; i < 4; i++) x[i] = __ldg(q + i);
  x[4] = sh ? __ldg(q + 4) : 0u;
#pragma unroll
  for (int i = 0; i < 4; i++) w[i] = __funnelshift_r(x[i], x[i + 1], sh);
}

// The direct path: entries written straight to global memory, one lane per
// entry, then the CRC read back from there.
__device__ __forceinline__ void enc_direct(const JobDev& J, const uint32_t* h5,
                                           const uint32_t* xinv, const uint32_t* tab8, uint64_t b,
                                           uint8_t* dst, uint32_t lane) {
  const uint64_t s = J.b_first[b], n = J.b_first[b + 1] - s;
  const uint32_t R = J.restart_interval;
  const uint32_t bsz = J.b_size[b];
  const uint64_t nrest = (n + R - 1) / R;
  uint8_t* ra = dst + bsz - 4 * nrest - 4;
  uint64_t carry = 0;
  for (uint64_t j0 = 0; j0 < n; j0 += 32) {
    const uint64_t j = j0 + lane;
    const bool valid = j < n;
    const bool restart = (j % R) == 0;
    const uint64_t k = s + j;
    const uint64_t size = valid ? (restart ? J.k_a[k] : J.k_b[k]) : 0;
    uint64_t tot;
    const uint64_t ex = warp_excl<uint64_t>(size, &tot) + carry;
    carry += tot;
    if (valid) {
      const uint32_t kl = J.k_klen[k], vl = J.k_vlen[k];
      const uint8_t* key = J.keys + J.k_koff[k];
      const uint8_t* val = J.in + J.k_voff[k];
      const uint32_t sh = restart ? 0 : J.k_shared[k];
      uint8_t* p = dst + ex;
      p = put_varint(p, sh);
      p = put_varint(p, kl - sh);
      p = put_varint(p, vl);
      if (J.dec_vpos)  // the value's place in its file, for the decoded form
        J.dec_vpos[k] = (uint32_t)(J.b_off[b] + (uint64_t)(p - dst) + (kl - sh));
      for (uint32_t i = sh; i < kl; i++) *p++ = key[i];
      for (uint32_t i = 0; i < vl; i++) *p++ = val[i];
      if (restart) {
        const uint64_t rem = n - j;
        const uint32_t cnt = (uint32_t)(rem < R ? rem : R);
        st_le32(ra + 4 * (j / R), ((uint32_t)ex << 8) | cnt);
      }
    }
  }
  if (lane == 0) {
    st_le32(dst + bsz - 4, (uint32_t)nrest);
    dst[bsz] = 0;
  }
  __syncwarp();
  const uint32_t crc = warp_block_crc_rows(h5, xinv, tab8, dst, bsz);
  if (lane == 0) st_le32(dst + bsz + 1, crc);
}

// A key delta or value of `len` bytes at stage position pos, from base +
// off.  A stretch shorter than kEncLong is staged whole; a longer one lists
// its whole 16-byte chunks in slot li while the list has room, and stages only
// its unaligned head and tail.  enc_list records the slot (li advances past
// every long stretch); enc_stage writes the staged bytes, and the chunks of a
// long stretch that found the list full.
__device__ __forceinline__ void enc_list(EncWarp& W, uint32_t pos, uint32_t len, uint32_t off,
                                         uint32_t from, uint32_t& li) {
  if (len < kEncLong) return;
  if (li < kEncMaxLong) {
    const uint32_t first = (pos + 15) & ~15u, last = (pos + len) & ~15u;
    W.ls_c0[li] = (first >> 4) | from;
    W.ls_n[li] = (last - first) >> 4;
    W.ls_src[li] = off + (first - pos);
  }
  li++;
}

__device__ __forceinline__ void enc_stage(uint8_t* st, uint32_t pos, uint32_t len,
                                          const uint8_t* src, bool listed) {
  if (len < kEncLong) {
    // the 16-byte form when every lane here has at most 16 bytes (a lane
    // that takes the 32-byte form is right for any length below kEncLong)
    if (__all_sync(__activemask(), len <= 16))
      copy_small<16>(st + pos, src, len);
    else
      copy_small<32>(st + pos, src, len);
    return;
  }
  const uint32_t first = (pos + 15) & ~15u, last = (pos + len) & ~15u;
  copy_small<16>(st + pos, src, first - pos);
  copy_small<16>(st + last, src + (last - pos), pos + len - last);
  if (!listed) {
    const uint32_t nq = (last - first) >> 4;
    for (uint32_t q = 0; q < nq; q++) {
      uint32_t w[4];
      load16(src + (first - pos) + 16 * q, w);
      *reinterpret_cast<uint4*>(st + first + 16 * q) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// A chunk slot: the five words holding a chunk's 16 bytes as loaded, and
// the right shift (bits) that aligns them.  Loads fill the slot; the shift is
// applied only where the chunk is used, so a slot loaded ahead does not hold
// up the warp until then.
struct EncSlot {
  uint32_t x[5];
  uint32_t sh;
};

__device__ __forceinline__ void enc_slot_load(const uint8_t* src, EncSlot& s) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  s.sh = 8 * (uint32_t)(a & 3);
#pragma unroll
  for (int i = 0; i < 4; i++) s.x[i] = __ldg(q + i);
  s.x[4] = s.sh ? __ldg(q + 4) : 0u;
}

// Chunk c of the stage grid from its source when it lies in listed stretch
// *k (k advances along the list); false when it is a stage chunk.
__device__ __forceinline__ bool enc_fetch_listed(const JobDev& J, const EncWarp& W, uint32_t nls,
                                                 uint32_t c, uint32_t& k, EncSlot& s) {
  while (k < nls && c >= (W.ls_c0[k] & ~kEncFromInput) + W.ls_n[k]) k++;
  const uint32_t c0 = k < nls ? W.ls_c0[k] : 0xffffffffu;
  if (c0 != 0xffffffffu && c >= (c0 & ~kEncFromInput)) {
    const uint8_t* base = (c0 & kEncFromInput) ? J.in : J.keys;
    enc_slot_load(base + W.ls_src[k] + 16 * (c - (c0 & ~kEncFromInput)), s);
    return true;
  }
  return false;
}

__device__ __forceinline__ void enc_fetch_stage(const uint8_t* st, uint32_t c, EncSlot& s) {
  const uint4 v = *reinterpret_cast<const uint4*>(st + 16 * c);
  s.x[0] = v.x, s.x[1] = v.y, s.x[2] = v.z, s.x[3] = v.w, s.x[4] = 0u;
  s.sh = 0u;
}

__device__ __forceinline__ void enc_fetch(const JobDev& J, const EncWarp& W, const uint8_t* st,
                                          uint32_t nls, uint32_t c, uint32_t& k, EncSlot& s) {
  if (!enc_fetch_listed(J, W, nls, c, k, s)) enc_fetch_stage(st, c, s);
}

// Chunk at stage position p out to global memory when it lies wholly inside
// the message [m0, m1) (block and type byte), and into the lane's CRC share.
// The grid bytes outside the message are zero in every chunk (the stage's
// edges are cleared), so every chunk takes the same step; the CRC's initial
// register is added at the end.
__device__ __forceinline__ void enc_chunk_out(const uint32_t* h5, uint8_t* gbase, uint32_t p,
                                              uint32_t m0, uint32_t m1, const EncSlot& s,
                                              uint32_t& u, uint32_t& last) {
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; i++) w[i] = __funnelshift_r(s.x[i], s.x[i + 1], s.sh);
  if (p >= m0 && p + 16 <= m1)
    *reinterpret_cast<uint4*>(gbase + p) = make_uint4(w[0], w[1], w[2], w[3]);
  u = crc_h5(h5, w[0] ^ u, w[1], w[2], w[3]);
  last = p;
}

// A block's place and entry range, loaded one block ahead; lane j's entry of
// its first 32 is copied to the warp's `ahead` area (cp.async, no registers
// held) while the current block is encoded, so that the next block's first
// steps do not wait on two rounds of dependent loads.
struct EncAhead {
  uint8_t* dst;
  uint32_t bsz, n;
  uint32_t s;
};

__device__ __forceinline__ void enc_ahead_entries(const JobDev& J, EncWarp& W, const EncAhead& A,
                                                  uint32_t lane) {
  cp_async_wait_all();  // no copy into the area is still in flight
  if (lane < A.n) {
    const uint32_t k = A.s + lane;
    cp_async4(&W.ahead[0][lane], J.k_klen + k);
    cp_async4(&W.ahead[1][lane], J.k_shared + k);
    cp_async4(&W.ahead[2][lane], J.k_vlen + k);
    cp_async4(&W.ahead[3][lane], J.k_koff + k);
    cp_async4(&W.ahead[4][lane], J.k_voff + k);
  }
}

// x / R for the restart interval R: a shift when R is a power of two (the
// common 16), else a division.
struct RestartDiv {
  uint32_t R, sh;
  bool pow2;
  __device__ __forceinline__ explicit RestartDiv(uint32_t r) {
    R = r;
    pow2 = (r & (r - 1u)) == 0u;
    sh = (uint32_t)__popc(r - 1u);  // log2 r when r is a power of two
  }
  __device__ __forceinline__ uint32_t div(uint32_t x) const {
    uint32_t q;
    if (pow2)
      q = x >> sh;
    else
      q = x / R;
    return q;
  }
  __device__ __forceinline__ bool starts_run(uint32_t x) const { return x - div(x) * R == 0u; }
};

__global__ void __launch_bounds__(kEncWarps * 32, 3) k_encode_blocks(const JobDev* __restrict__ jobs) {
  __shared__ uint32_t s_h5[kCrcH5Words];
  __shared__ uint32_t s_xinv[kCrcXinvSmem];
  __shared__ uint32_t s_tab8[256];
  __shared__ JobDev s_job;  // the job's descriptor, read from here in every step
  extern __shared__ __align__(16) uint8_t enc_smem[];
  copy_job(jobs + blockIdx.y, &s_job);
  const JobDev& G = jobs[blockIdx.y];
  for (uint32_t i = threadIdx.x; i < kCrcH5Words; i += blockDim.x) s_h5[i] = G.crc_h5[i];
  for (uint32_t i = threadIdx.x; i < kCrcXinvN; i += blockDim.x) s_xinv[xinv_slot(i)] = G.crc_xinv[i];
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) s_tab8[i] = G.crc_byte[i];
  __syncthreads();
  const JobDev& J = s_job;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  EncWarp& W = reinterpret_cast<EncWarp*>(enc_smem)[warp];
  if (J.ctr->error) return;
  const uint32_t nb = (uint32_t)J.ctr->n_blocks_out;  // block and survivor indices fit 32 bits
  const uint32_t R = J.restart_interval;
  const RestartDiv rd(R);
  const uint32_t stride = gridDim.x * kEncWarps;
  uint8_t* st = W.stage;
  uint32_t b = blockIdx.x * kEncWarps + warp;
  EncAhead cur{};
  if (b < nb) {
    cur.dst = J.out + J.files[J.b_file[b]].out_off + J.b_off[b];
    cur.bsz = J.b_size[b];
    cur.s = J.b_first[b];
    cur.n = (uint32_t)(J.b_first[b + 1] - cur.s);
    enc_ahead_entries(J, W, cur, lane);
  }
  for (; b < nb; b += stride) {
    // the next block's place and range (its entries follow after step 2)
    const uint32_t bn = b + stride;
    EncAhead nxt{};
    uint32_t n_file = 0;
    uint64_t n_off = 0;
    if (bn < nb) {
      n_file = J.b_file[bn];
      n_off = J.b_off[bn];
      nxt.bsz = J.b_size[bn];
      nxt.s = J.b_first[bn];
      nxt.n = (uint32_t)(J.b_first[bn + 1] - nxt.s);
    }
    uint8_t* dst = cur.dst;
    const uint32_t bsz = cur.bsz, n = cur.n;
    const uint32_t s = cur.s;
    const uint32_t ph = (uint32_t)(reinterpret_cast<uintptr_t>(dst) & 15);
    if (ph + bsz + kTrailer + 16 > kEncStage) {
      enc_direct(J, s_h5, s_xinv, s_tab8, b, dst, lane);
    } else {
      const uint32_t nrest = rd.div(n + R - 1);
      const uint32_t rbase = ph + bsz - 4 * nrest - 4;  // stage position of the restart array
      const uint32_t m0 = ph, m1 = ph + bsz + 1;        // the message: block and type byte
      // the initial register's share of the CRC, and zeros in the stage's
      // first and last chunks (grid bytes outside the message)
      const uint32_t ones = __ldg(J.crc_ones + (m1 - m0));
      if (lane == 0) *reinterpret_cast<uint4*>(st) = make_uint4(0u, 0u, 0u, 0u);
      if (lane == 1) *reinterpret_cast<uint4*>(st + ((m1 - 1) & ~15u)) = make_uint4(0u, 0u, 0u, 0u);
      __syncwarp();
      // 1. entries: the long stretches listed first; once the list is
      // complete (last round) the first two chunk rows' listed chunks are
      // loaded while the lanes write headers, restart words, short stretches
      // and cut edges to the stage
      uint32_t carry = 0, lcarry = 0, nls = 0, k = 0;
      EncSlot sa{}, sb{};
      bool ga = false, gb = false;  // sa / sb came from a listed stretch
      for (uint32_t j0 = 0; j0 < n; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t size = 0, hl = 0, kd = 0, vl = 0, sh = 0, koff = 0, voff = 0;
        if (j < n) {
          uint32_t kl;
          if (j0 == 0) {
            cp_async_wait_all();  // this lane's own copies
            kl = W.ahead[0][lane], sh = W.ahead[1][lane], vl = W.ahead[2][lane];
            koff = W.ahead[3][lane], voff = W.ahead[4][lane];
          } else {
            const uint32_t e = s + j;
            kl = J.k_klen[e], sh = J.k_shared[e], vl = J.k_vlen[e];
            koff = J.k_koff[e], voff = J.k_voff[e];
          }
          if (rd.starts_run(j)) sh = 0;
          kd = kl - sh;
          koff += sh;
          hl = varint_len32(sh) + varint_len32(kd) + varint_len32(vl);
          size = hl + kd + vl;
        }
        uint32_t tot, ltot;
        const uint32_t ex = warp_excl<uint32_t>(size, &tot) + carry;
        const uint32_t nl = j < n ? (uint32_t)(kd >= kEncLong) + (uint32_t)(vl >= kEncLong) : 0u;
        uint32_t li = warp_excl<uint32_t>(nl, &ltot) + lcarry;
        carry += tot;
        lcarry += ltot;
        const uint32_t kpos = ph + ex + hl;
        const uint32_t lik = li;
        if (j < n) enc_list(W, kpos, kd, koff, 0u, li);
        const uint32_t liv = li;
        if (j < n) enc_list(W, kpos + kd, vl, voff, kEncFromInput, li);
        if (j0 + 32 >= n) {
          __syncwarp();
          nls = min(lcarry, kEncMaxLong);
          if (16 * lane < m1) ga = enc_fetch_listed(J, W, nls, lane, k, sa);
          if (16 * (lane + 32) < m1) gb = enc_fetch_listed(J, W, nls, lane + 32, k, sb);
        }
        if (j < n) {
          uint8_t* p = st + ph + ex;
          p = put_varint32(p, sh);
          p = put_varint32(p, kd);
          put_varint32(p, vl);
          const uint32_t run = rd.div(j);
          if (j == run * R) {
            const uint32_t rem = n - j;
            st_le32(st + rbase + 4 * run, (ex << 8) | (rem < R ? rem : R));
          }
          if (J.dec_vpos)  // the value's place in its file, for the decoded form
            J.dec_vpos[s + j] = (uint32_t)(J.b_off[b] + ex + hl + kd);
          enc_stage(st, kpos, kd, J.keys + koff, lik < kEncMaxLong);
          enc_stage(st, kpos + kd, vl, J.in + voff, liv < kEncMaxLong);
        }
      }
      if (lane == 0) {
        st_le32(st + ph + bsz - 4, nrest);
        st[ph + bsz] = 0;  // kNoCompression
      }
      __syncwarp();
      // 2. chunks: out to global memory and into the CRC; each chunk's loads
      // are issued two chunks ahead of its use (three rotating slots)
      uint8_t* gbase = dst - ph;
      uint32_t u = 0, last = 0xffffffffu;
      EncSlot sc;
      bool vb = 16 * (lane + 32) < m1;
      if (16 * lane < m1 && !ga) enc_fetch_stage(st, lane, sa);
      if (vb && !gb) enc_fetch_stage(st, lane + 32, sb);
      if (bn < nb) {  // the next block's place and entries, in flight meanwhile
        nxt.dst = J.out + J.files[n_file].out_off + n_off;
        enc_ahead_entries(J, W, nxt, lane);
      }
      for (uint32_t c = lane; 16 * c < m1; c += 96) {
        const bool vc = 16 * (c + 64) < m1;
        if (vc) enc_fetch(J, W, st, nls, c + 64, k, sc);
        enc_chunk_out(s_h5, gbase, 16 * c, m0, m1, sa, u, last);
        if (16 * (c + 96) < m1) enc_fetch(J, W, st, nls, c + 96, k, sa);
        if (vb) enc_chunk_out(s_h5, gbase, 16 * (c + 32), m0, m1, sb, u, last);
        const bool ve = 16 * (c + 128) < m1;
        if (ve) enc_fetch(J, W, st, nls, c + 128, k, sb);
        if (vc) enc_chunk_out(s_h5, gbase, 16 * (c + 64), m0, m1, sc, u, last);
        vb = ve;
      }
      // the lines the next block's entry pass copies bytes from (its keys,
      // its values' first and last bytes) into L2 while this block finishes
      if (bn < nb && lane < nxt.n) {
        cp_async_wait_all();
        const uint32_t pkl = W.ahead[0][lane], pvl = W.ahead[2][lane];
        const uint32_t pko = W.ahead[3][lane], pvo = W.ahead[4][lane];
        prefetch_l2(J.keys + pko);
        prefetch_l2(J.keys + pko + pkl - 1);
        prefetch_l2(J.in + pvo);
        if (pvl) prefetch_l2(J.in + pvo + pvl - 1);
      }
      // 3. CRC (with the initial register's share), trailer, partial chunks
      // at both ends
      const uint32_t full = crc_rows_raw(s_xinv, s_tab8, u, last, m1) ^ ones ^ 0xffffffffu;
      const uint32_t crc = ((full >> 15) | (full << 17)) + 0xa282ead8u;  // crc32c::Mask
      if (lane == 0) st_le32(st + m1, crc);
      __syncwarp();
      const uint32_t cf0 = (m0 + 15) >> 4, cf1 = m1 >> 4;  // whole chunks [cf0, cf1) went out
      uint32_t h1 = 16 * cf0, t0 = 16 * cf1;
      if (cf1 < cf0) h1 = t0 = m0;  // the message lies inside one chunk
      const uint32_t nh = h1 - m0, nt = m1 + 4 - t0;
      for (uint32_t x = lane; x < nh + nt; x += 32) {
        const uint32_t q = x < nh ? m0 + x : t0 + (x - nh);
        gbase[q] = st[q];
      }
      __syncwarp();
    }
    if (bn < nb && nxt.dst == nullptr) {  // the direct path
      nxt.dst = J.out + J.files[n_file].out_off + n_off;
      enc_ahead_entries(J, W, nxt, lane);
    }
    cur = nxt;
  }
  cp_async_wait_all();  // a direct-path last block never waited for its entries' copies
}

// The survivors' decoded form for later jobs (keep_decoded): key bytes at
// dec_kcum (a scan of the key lengths), value lengths, prefixes and tags; the
// value places were written by k_encode_blocks.  One warp per 32 survivors,
// lanes over the group's key bytes.
__global__ void k_emit_decoded(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error || !J.dec_keys) return;
  const uint64_t n = J.ctr->n_kept;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g * 32 < n; g += warps) {
    const uint64_t k = g * 32 + lane;
    if (k < n) {
      uint32_t kl;
      const uint8_t* key = kept_key(J, k, &kl);
      J.dec_vlen[k] = J.k_vlen[k];
      J.dec_pfx[k] = user_prefix(key, kl);
      J.dec_tag[k] = ld_le64(key + kl - 8);
    }
    const uint64_t k1 = min(n, g * 32 + 32);
    for (uint64_t j = g * 32; j < k1; j++) {
      uint32_t kl;
      const uint8_t* key = kept_key(J, j, &kl);
      uint8_t* d = J.dec_keys + J.dec_kcum[j];
      for (uint32_t t = lane; t < kl; t += 32) d[t] = key[t];
    }
  }
}

// One warp per filter group (at the group's first block).  The bloom bits are
// set with shared-memory atomics in the warp's buffer `sbuf` (kFilterSmem
// bytes) and written out with coalesced byte stores; larger filters are built
// in place with global atomics.
constexpr uint32_t kFilterSmem = 1024;
__device__ __forceinline__ void encode_filter_group(const JobDev& J, uint64_t b, uint32_t lane,
                                                    uint32_t* sbuf) {
  const FileOut& F = J.files[J.b_file[b]];
  const uint32_t fb0 = F.first_block, fb1 = F.end_block;
  uint8_t* fbase = J.out + F.out_off + F.filter_off;
  const uint64_t Ft = J.b_gcum[fb1] - J.b_gcum[fb0];
  const uint32_t gb = J.b_gbytes[b];
  if (gb != 0) {
    uint8_t* fdst = fbase + (J.b_gcum[b] - J.b_gcum[fb0]);
    const uint32_t nbytes = gb - 1;
    const uint32_t bits = nbytes * 8;  // a group's filter is far below 2^29 bytes
    const bool in_smem = nbytes <= kFilterSmem;
    if (in_smem) {
      for (uint32_t i = lane; i < (nbytes + 3) / 4; i += 32) sbuf[i] = 0;
    } else {
      for (uint32_t i = lane; i < nbytes; i += 32) fdst[i] = 0;
    }
    __syncwarp();
    const uint64_t k0 = J.b_first[b];
    const uint32_t nk = J.b_gkeys[b];
    const FastMod mod(bits);
    for (uint32_t i = lane; i < nk; i += 32) {
      uint32_t kl;
      const uint8_t* key = kept_key(J, k0 + i, &kl);
      uint32_t h = leveldb_hash_words(key, kl - 8, 0xbc9f1d34u);
      const uint32_t delta = (h >> 17) | (h << 15);
      for (uint32_t q = 0; q < J.bloom_k; q++) {
        const uint32_t bitpos = mod(h);
        if (in_smem) {
          // byte bitpos/8, bit bitpos%8 = bit (bitpos & 31) of little-endian word bitpos/32
          atomicOr(&sbuf[bitpos >> 5], 1u << (bitpos & 31));
        } else {
          uint8_t* byte = fdst + (bitpos >> 3);
          const uintptr_t a = reinterpret_cast<uintptr_t>(byte);
          unsigned int* word = reinterpret_cast<unsigned int*>(a & ~uintptr_t(3));
          atomicOr(word, 1u << ((a & 3) * 8 + (bitpos & 7)));
        }
        h += delta;
      }
    }
    __syncwarp();
    if (in_smem) {
      const uint8_t* sb = reinterpret_cast<const uint8_t*>(sbuf);
      for (uint32_t i = lane; i < nbytes; i += 32) fdst[i] = sb[i];
      __syncwarp();
    }
    if (lane == 0) fdst[nbytes] = (uint8_t)J.bloom_k;
    // filter offsets of the empty indices before this group and of the group
    const uint64_t jb = J.b_off[b] >> kFilterBaseLg;
    const int64_t jprev = (b == fb0) ? -1 : (int64_t)(J.b_off[b - 1] >> kFilterBaseLg);
    const uint32_t val = (uint32_t)(J.b_gcum[b] - J.b_gcum[fb0]);
    for (int64_t jj = jprev + 1 + lane; jj <= (int64_t)jb; jj += 32)
      st_le32(fbase + Ft + 4 * jj, val);
  }
}

// A filter group of at most kFilterThreadKeys keys whose filter has at most
// kFilterLocal bytes, by one thread: the bits in a thread-local array, then
// byte stores.  Groups of more keys are built by a warp.
constexpr uint32_t kFilterLocal = 128;
constexpr uint32_t kFilterThreadKeys = 8;
__device__ __forceinline__ void filter_group_thread(const JobDev& J, uint64_t b, uint32_t gb) {
  const FileOut& F = J.files[J.b_file[b]];
  const uint32_t fb0 = F.first_block, fb1 = F.end_block;
  uint8_t* fbase = J.out + F.out_off + F.filter_off;
  const uint64_t Ft = J.b_gcum[fb1] - J.b_gcum[fb0];
  uint8_t* fdst = fbase + (J.b_gcum[b] - J.b_gcum[fb0]);
  const uint32_t nbytes = gb - 1;
  const uint32_t bits = nbytes * 8;
  uint32_t w[kFilterLocal / 4];
#pragma unroll
  for (uint32_t i = 0; i < kFilterLocal / 4; i++) w[i] = 0;
  const uint64_t k0 = J.b_first[b];
  const uint32_t nk = J.b_gkeys[b];
  const FastMod mod(bits);
  for (uint32_t i = 0; i < nk; i++) {
    uint32_t kl;
    const uint8_t* key = kept_key(J, k0 + i, &kl);
    uint32_t h = leveldb_hash_words(key, kl - 8, 0xbc9f1d34u);
    const uint32_t delta = (h >> 17) | (h << 15);
    for (uint32_t q = 0; q < J.bloom_k; q++) {
      const uint32_t bitpos = mod(h);
      w[bitpos >> 5] |= 1u << (bitpos & 31);  // byte bitpos/8, bit bitpos%8
      h += delta;
    }
  }
  for (uint32_t i = 0; i < nbytes; i++) fdst[i] = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
  fdst[nbytes] = (uint8_t)J.bloom_k;
  // filter offsets of the empty indices before this group and of the group
  const uint64_t jb = J.b_off[b] >> kFilterBaseLg;
  const int64_t jprev = (b == fb0) ? -1 : (int64_t)(J.b_off[b - 1] >> kFilterBaseLg);
  const uint32_t val = (uint32_t)(J.b_gcum[b] - J.b_gcum[fb0]);
  for (int64_t jj = jprev + 1; jj <= (int64_t)jb; jj++) st_le32(fbase + Ft + 4 * jj, val);
}

// Filter groups (at their first blocks): groups of a few keys one per thread,
// larger ones one per warp (bits in the warp's shared memory, or in place).
__global__ void k_encode_filters(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_filter[8][kFilterSmem / 4];  // blockDim 256: 8 warps
  const uint32_t lane = threadIdx.x & 31;
  if (J.bits_per_key <= 0 || J.ctr->error) return;
  const uint64_t nb = J.ctr->n_blocks_out;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t gb = J.b_gbytes[b];
    if (gb != 0 && J.b_gkeys[b] <= kFilterThreadKeys && gb - 1 <= kFilterLocal)
      filter_group_thread(J, b, gb);
  }
  // the larger groups: warp w takes blocks w, w + W, w + 2W, ... (W warps in
  // all), looking at 32 of them with one load per lane and building the ones
  // that need it
  const uint64_t W = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint64_t b0 = w; b0 < nb; b0 += 32 * W) {
    const uint64_t b = b0 + lane * W;
    bool big = false;
    if (b < nb) {
      const uint32_t gb = J.b_gbytes[b];
      big = gb != 0 && (J.b_gkeys[b] > kFilterThreadKeys || gb - 1 > kFilterLocal);
    }
    for (unsigned m = __ballot_sync(0xffffffffu, big); m; m &= m - 1)
      encode_filter_group(J, b0 + (uint64_t)(__ffs(m) - 1) * W, lane, s_filter[threadIdx.x >> 5]);
  }
}

__device__ __forceinline__ void encode_index_entry(const JobDev& J, uint64_t b) {
  const FileOut& F = J.files[J.b_file[b]];
  const uint32_t fb0 = F.first_block, fb1 = F.end_block;
  uint8_t* ib = J.out + F.out_off + F.index_off;
  const uint64_t eoff = J.b_icum[b] - J.b_icum[fb0];
  uint8_t* p = ib + eoff;
  const uint32_t ilen = J.b_ilen[b], sep = J.b_sep[b];
  const uint64_t off = J.b_off[b];
  const uint32_t bsz = J.b_size[b];
  *p++ = 0;
  p = put_varint(p, ilen);
  p = put_varint(p, varint_len(off) + varint_len(bsz));
  uint32_t llen;
  const uint8_t* lkey = kept_key(J, J.b_first[b + 1] - 1, &llen);
  if (sep == kNoSep) {
    for (uint32_t i = 0; i < ilen; i++) p[i] = lkey[i];
  } else {
    for (uint32_t i = 0; i < sep; i++) p[i] = lkey[i];
    p[sep] = (uint8_t)(lkey[sep] + 1);
    uint64_t t = kSeekTag;
    for (int i = 0; i < 8; i++) p[sep + 1 + i] = (uint8_t)(t >> (8 * i));
  }
  p += ilen;
  p = put_varint(p, off);
  p = put_varint(p, bsz);
  uint8_t* ra = ib + (J.b_icum[fb1] - J.b_icum[fb0]) + 4 * (b - fb0);
  st_le32(ra, ((uint32_t)eoff << 8) | 1u);
  if (b + 1 == fb1) st_le32(ra + 4, fb1 - fb0);
}

__global__ void k_encode_index(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;
  const uint64_t nb = J.ctr->n_blocks_out;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x)
    encode_index_entry(J, b);
}

// Metaindex, footer and the tail of the filter block's offset array (thread
// 0), then the trailers of the filter, metaindex and index blocks, each a
// CRC32C over the whole CTA: one CTA per output file.
__global__ void __launch_bounds__(256) k_encode_meta(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_skip;
  if (threadIdx.x == 0) s_skip = J.ctr->error || blockIdx.x >= J.ctr->n_files;
  __syncthreads();
  if (s_skip) return;
  const uint32_t f = blockIdx.x;
  if (threadIdx.x == 0) {
    const FileOut& F = J.files[f];
    uint8_t* base = J.out + F.out_off;
    if (J.bits_per_key > 0) {
      uint8_t* fb = base + F.filter_off;
      const uint64_t Ft = J.b_gcum[F.end_block] - J.b_gcum[F.first_block];
      const uint64_t jlast = J.b_off[F.end_block - 1] >> kFilterBaseLg;
      for (uint64_t jj = jlast + 1; jj < F.n_filters; jj++) st_le32(fb + Ft + 4 * jj, (uint32_t)Ft);
      st_le32(fb + Ft + 4ull * F.n_filters, (uint32_t)Ft);
      fb[Ft + 4ull * F.n_filters + 4] = (uint8_t)kFilterBaseLg;
      uint8_t* m = base + F.meta_off;
      m[0] = 0;
      m[1] = (uint8_t)kFilterNameLen;
      m[2] = (uint8_t)(varint_len(F.filter_off) + varint_len(F.filter_size));
      for (uint32_t i = 0; i < kFilterNameLen; i++) m[3 + i] = (uint8_t)kFilterName[i];
      uint8_t* p = m + 3 + kFilterNameLen;
      p = put_varint(p, F.filter_off);
      p = put_varint(p, F.filter_size);
      st_le32(p, 1u);  // restart word (0 << 8) | 1
      st_le32(p + 4, 1u);
    } else {
      uint8_t* m = base + F.meta_off;
      st_le32(m, 0u);
      st_le32(m + 4, 1u);
    }
    uint8_t* foot = base + F.size - kFooter;
    for (int i = 0; i < 40; i++) foot[i] = 0;
    uint8_t* p = foot;
    p = put_varint(p, F.meta_off);
    p = put_varint(p, F.meta_size);
    p = put_varint(p, F.index_off);
    p = put_varint(p, F.index_size);
    st_le32(foot + 40, 0x8b80fb57u);
    st_le32(foot + 44, 0xdb477524u);
  }
  __syncthreads();
  const FileOut& F = J.files[f];
  // the file's smallest and largest internal keys (FileMetaData::smallest /
  // largest) into slots 2f and 2f + 1 of fkey_stride bytes, their lengths
  // into fkoff; every key fits a slot (a single-pass job with a longer key
  // was rerun with exact counting, whose stride is the longest key)
  for (uint32_t which = 0; which < 2; which++) {
    uint32_t l;
    const uint8_t* k = kept_key(J, which ? F.end_kept - 1 : F.first_kept, &l);
    uint8_t* d = J.fkeys + (2ull * f + which) * J.fkey_stride;
    for (uint32_t t = threadIdx.x; t < l; t += blockDim.x) d[t] = k[t];
    if (threadIdx.x == 0) J.fkoff[2 * f + which] = l;
  }
}

// The filter, metaindex and index blocks' trailers: each region is cut into
// kMetaPiece-byte pieces, one warp per piece (the row CRC, lanes over the
// piece's 16-byte chunks); a piece's raw register, moved to the region's end
// past its type byte, is xored into the file's accumulator (the xor of every
// byte's share is the register of the whole), and k_meta_trailers writes the
// finished CRCs.  CTAs per file: from the entries per file (the filter and
// index blocks grow with them), 4 to 32.
constexpr uint32_t kMetaPiece = 4096;

__device__ __forceinline__ void meta_region(const FileOut& F, uint32_t r, uint64_t* off,
                                            uint64_t* len) {
  if (r == 0) {
    *off = F.filter_off;
    *len = F.filter_size;
  } else if (r == 1) {
    *off = F.meta_off;
    *len = F.meta_size;
  } else {
    *off = F.index_off;
    *len = F.index_size;
  }
}

__global__ void __launch_bounds__(256) k_meta_crc(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.z];
  __shared__ uint32_t s_h5[kCrcH5Words];
  __shared__ uint32_t s_xinv[kCrcXinvSmem];
  __shared__ uint32_t s_tab8[256];
  __shared__ uint32_t s_skip;
  if (threadIdx.x == 0) s_skip = J.ctr->error || blockIdx.y >= J.ctr->n_files;
  for (uint32_t i = threadIdx.x; i < kCrcH5Words; i += blockDim.x) s_h5[i] = J.crc_h5[i];
  for (uint32_t i = threadIdx.x; i < kCrcXinvN; i += blockDim.x) s_xinv[xinv_slot(i)] = J.crc_xinv[i];
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) s_tab8[i] = J.crc_byte[i];
  __syncthreads();
  if (s_skip) return;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t nf = J.ctr->n_files;
  for (uint32_t f = blockIdx.y; f < nf; f += gridDim.y) {
    const FileOut& F = J.files[f];
    uint64_t off[3], len[3], np[3];
    for (uint32_t r = 0; r < 3; r++) {
      meta_region(F, r, &off[r], &len[r]);
      np[r] = (r == 0 && J.bits_per_key <= 0) ? 0 : (len[r] + kMetaPiece - 1) / kMetaPiece;
    }
    const uint8_t* fbase = J.out + F.out_off;
    const uint64_t total = np[0] + np[1] + np[2];
    for (uint64_t p = (uint64_t)blockIdx.x * (blockDim.x / 32) + warp; p < total;
         p += (uint64_t)gridDim.x * (blockDim.x / 32)) {
      uint32_t r = 0;
      uint64_t q = p;
      while (q >= np[r]) q -= np[r++];
      const uint64_t a = q * kMetaPiece, e = min(len[r], a + kMetaPiece);
      const uint8_t* pa = fbase + off[r] + a;
      const uint32_t m0 = (uint32_t)(reinterpret_cast<uintptr_t>(pa) & 15);
      const uint32_t m1 = m0 + (uint32_t)(e - a);
      const uint8_t* g = pa - m0;
      // the lane's chunks of the piece, all loaded before the CRC steps
      constexpr uint32_t kRows = (kMetaPiece + 15) / kCrcRowBytes + 1;
      uint4 v[kRows];
#pragma unroll
      for (uint32_t i = 0; i < kRows; i++) {
        const uint32_t x = 16 * lane + kCrcRowBytes * i;
        if (x < m1) v[i] = *reinterpret_cast<const uint4*>(g + x);
      }
      uint32_t u = 0, last = 0xffffffffu;
#pragma unroll
      for (uint32_t i = 0; i < kRows; i++) {
        const uint32_t x = 16 * lane + kCrcRowBytes * i;
        if (x < m1) {
          u = crc_chunk_step(s_h5, u, x, m0, m1, v[i].x, v[i].y, v[i].z, v[i].w, a == 0);
          last = x;
        }
      }
      const uint32_t raw = crc_rows_raw(s_xinv, s_tab8, u, last, m1);
      if (lane == 0)
        atomicXor(&J.files[f].crc_acc[r], crc_shift_tab(J, s_tab8, raw, len[r] + 1 - e));
    }
  }
}

__global__ void k_meta_trailers(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;
  const uint32_t nf = J.ctr->n_files;
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < 3 * nf; x += gridDim.x * blockDim.x) {
    const uint32_t f = x / 3, r = x % 3;
    if (r == 0 && J.bits_per_key <= 0) continue;
    const FileOut& F = J.files[f];
    uint64_t off, len;
    meta_region(F, r, &off, &len);
    uint8_t* p = J.out + F.out_off + off + len;
    const uint32_t full = F.crc_acc[r] ^ 0xffffffffu;
    p[0] = 0;  // kNoCompression
    st_le32(p + 1, ((full >> 15) | (full << 17)) + 0xa282ead8u);  // crc32c::Mask
  }
}

inline unsigned per_job(const Batch& bt, unsigned total) {
  return bt.ctas_per_job ? bt.ctas_per_job : std::max<unsigned>(1, total / bt.B);
}

}  // namespace

void launch_sizes(const Batch& bt, cudaStream_t st) {
  note_launch(), k_sizes<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B), 256, 0,
                           st>>>(bt.d);
}
void launch_next(const Batch& bt, cudaStream_t st) {
  note_launch(), k_next<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B), 256, 0,
                          st>>>(bt.d);
}
void launch_chain(const Batch& bt, cudaStream_t st) {
  const uint64_t chunks = (bt.max_entries + bt.chunk - 1) / bt.chunk + 1;
  // next() values, sub-chunk exits (windows up to kChainSub) and entry points
  const size_t smem = ((size_t)bt.chunk + (bt.chunk / kChainSub) * (kChainSub + 1)) * sizeof(uint32_t);
  const unsigned g = (unsigned)std::min<uint64_t>(chunks, per_job(bt, 148 * 4));
  note_launch(), k_chain_tables<<<dim3(g, bt.B), 256, smem, st>>>(bt.d);
  if (chunks > kChainGroup)
    note_launch(), k_chain_groups<<<dim3(grid_x(chunks / kChainGroup * bt.chunk, 256, 148 * 4), bt.B),
                                    256, 0, st>>>(bt.d);
  note_launch(), k_chain_resolve<<<dim3(1, bt.B), 1024, (size_t)bt.chain_smem_words * 4, st>>>(bt.d);
  note_launch(), k_chain_mark<<<dim3(g, bt.B), 128, smem, st>>>(bt.d);
}
void launch_block_list(const Batch& bt, cudaStream_t st) {
  note_launch(), k_block_list<<<dim3(grid_x(bt.max_entries + 1, 256, per_job(bt, 148 * 8)), bt.B), 256,
                                0, st>>>(bt.d);
}
void launch_files(const Batch& bt, cudaStream_t st) {
  note_launch(), k_forced_blocks<<<dim3((bt.max_cap_triggers + 255) / 256, bt.B), 256, 0, st>>>(bt.d);
  note_launch(), k_file_next<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B), 256, 0,
                               st>>>(bt.d);
  note_launch(), k_files<<<dim3(1, bt.B), kFileThreads, 0, st>>>(bt.d);
}
void launch_block_layout(const Batch& bt, cudaStream_t st) {
  note_launch(), k_block_layout<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B), 256,
                                  0, st>>>(bt.d);
}
void launch_file_layout(const Batch& bt, cudaStream_t st) {
  note_launch(), k_file_layout<<<dim3(1, bt.B), 256, 0, st>>>(bt.d);
}
void encode_kernel_attributes() {
  cudaFuncSetAttribute(k_encode_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEncSmem);
}

void launch_encode_blocks(const Batch& bt, cudaStream_t st) {
  // grid-stride over the device-side block count: 3 CTAs per SM x 4 waves,
  // shared out among the jobs
  note_launch(), k_encode_blocks<<<dim3(grid_x(bt.max_entries, kEncWarps, per_job(bt, 148 * 3 * 4)),
                                        bt.B), kEncWarps * 32, kEncSmem, st>>>(bt.d);
}
void launch_emit_decoded(const Batch& bt, cudaStream_t st) {
  if (!bt.any_keep_decoded) return;
  scan_batch(kScanDecKey, bt, bt.max_entries, st);
  note_launch(), k_emit_decoded<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B), 256,
                                  0, st>>>(bt.d);
}
void launch_encode_filters(const Batch& bt, cudaStream_t st) {
  note_launch(), k_encode_filters<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 8)), bt.B),
                                    256, 0, st>>>(bt.d);
}
void launch_encode_index(const Batch& bt, cudaStream_t st) {
  note_launch(), k_encode_index<<<dim3(grid_x(bt.max_entries, 256, per_job(bt, 148 * 16)), bt.B), 256,
                                  0, st>>>(bt.d);
}
void launch_encode_meta(const Batch& bt, cudaStream_t st) {
  note_launch(), k_encode_meta<<<dim3(bt.max_cap_files, bt.B), 256, 0, st>>>(bt.d);
  uint32_t per_file = 4;
  while (per_file < 32 && (uint64_t)per_file * 8192 * std::max<uint32_t>(bt.max_cap_files, 1) <
                              bt.max_entries)
    per_file *= 2;
  note_launch(), k_meta_crc<<<dim3(per_file, std::min<uint32_t>(bt.max_cap_files, 65535), bt.B),
                              256, 0, st>>>(bt.d);
  note_launch(), k_meta_trailers<<<dim3((3 * bt.max_cap_files + 255) / 256, bt.B), 256, 0, st>>>(bt.d);
}

}  // namespace lc
