// Merge and drop: decoded runs -> survivors in output order.
//
// * Merge: the reference merges its children with MergingIterator
//   (table/merger.cc:148, linear FindSmallest; on equal keys the earlier child
//   wins).  Here the children are merged pairwise in rounds with merge path,
//   in tiles: one thread per tile finds the tile's split by binary search,
//   then a CTA stages the tile's two stretches (entry ids and their 8-byte
//   user-key prefixes) in shared memory, merges them there (each thread its
//   own diagonal) and writes ids, prefixes and tags back coalesced, so that a
//   round reads and writes 20 bytes per entry and key bytes are read only for
//   equal prefixes.  Ties go to the left (earlier) group, which keeps child
//   order.  The drop rule then reads prefixes and tags in merged order.
// * Drop rule (db/db_impl.cc:1113-1147): an entry is hidden when the previous
//   entry has the same user key and a sequence number <= smallest_snapshot;
//   a deletion marker is dropped when its sequence number is <=
//   smallest_snapshot and no file at a level >= L+2 covers its user key
//   (Compaction::IsBaseLevelForKey, db/version_set.cc:1535-1554).  Keys whose
//   type byte is not 0/1 (ParseInternalKey fails) are kept and reset the state.
// * Grandparent cuts (Compaction::ShouldStopBefore, db/version_set.cc:
//   1556-1579): evaluated for every merged key, dropped or not.  The number of
//   grandparents whose largest key precedes each merged key is found by binary
//   search; the cut positions are then a chain of threshold searches over the
//   running overlap, which one thread resolves.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "lc_device.cuh"
#include "lc_kernels.h"

namespace lc {

namespace {

// The user-key bytes every input key of the job shares: the common prefix
// of the first and last keys of every merge child (each child is sorted, so
// its keys share what its two ends share) with the first key of child 0.
// Then, per grandparent, its prefix after those bytes, or where it sorts
// against every entry when it does not share them.  One CTA per job.
__global__ void k_key_skip(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed, s_skip;
  if (threadIdx.x == 0) {
    s_failed = J.ctr->error;
    s_skip = 0xffffffffu;
  }
  __syncthreads();
  if (s_failed) return;
  const uint64_t n = J.ctr->n_entries_in;
  uint32_t u0 = 0;
  const uint8_t* k0 = nullptr;
  if (n > 0) {
    k0 = J.keys + J.e_koff[0];
    u0 = J.e_klen[0] - 8;
  }
  // boundary keys: 2 per child
  for (uint32_t x = threadIdx.x; x < 2 * J.n_runs && n > 0; x += blockDim.x) {
    const uint32_t r = x >> 1;
    const uint64_t a = J.run_entry_begin[r], z = J.run_entry_begin[r + 1];
    if (a == z) continue;
    const uint64_t e = (x & 1) ? z - 1 : a;
    const uint8_t* k = J.keys + J.e_koff[e];
    const uint32_t u = J.e_klen[e] - 8, m = min(u, u0);
    uint32_t l = 0;
    while (l < m && k[l] == k0[l]) l++;
    atomicMin(&s_skip, l);
  }
  __syncthreads();
  const uint32_t L = n > 0 ? min(s_skip, u0) : 0;
  if (threadIdx.x == 0) J.ctr->key_skip = L;
  for (uint32_t g = threadIdx.x; g < J.n_gp; g += blockDim.x) {
    const uint64_t go = J.gp_key_off[g];
    const uint8_t* gk = J.gp_keys + go;
    const uint32_t gu = (uint32_t)(J.gp_key_off[g + 1] - go) - 8;
    uint32_t i = 0;
    const uint32_t m = min(gu, L);
    while (i < m && gk[i] == k0[i]) i++;
    uint8_t mode = 0;
    if (i < L) {
      // differs within the common bytes, or ends inside them: it sorts
      // before every entry (1) or after every entry (2)
      mode = (i == gu || gk[i] < k0[i]) ? 1 : 2;
    }
    J.gp_mode[g] = mode;
    J.gp_upfx[g] = mode ? 0 : user_prefix_after(gk, gu + 8, L);
  }
}

// True when entry e is the first of its merge child.
__device__ __forceinline__ bool run_first(const JobDev& J, uint64_t e) {
  // the last child whose first entry is at or before e
  uint32_t lo = 0, hi = J.n_runs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (J.run_entry_begin[mid] <= e) lo = mid;
    else hi = mid;
  }
  return J.run_entry_begin[lo] == e;
}

// e_pfx after the job's common bytes (the decode wrote the prefixes from the
// keys' first byte), and a check of the merge children's order: every key
// starts with the common bytes and sorts at or after the entry before it in
// its child.  table/merger.cc merges children it trusts to be sorted; a child
// out of order fails the job here (kErrUnsorted) rather than reaching the
// merge path, whose cuts assume sorted children.
__global__ void k_prefix(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;
  const uint32_t L = J.ctr->key_skip;
  const uint64_t n = J.ctr->n_entries_in;
  if (n == 0) return;
  const uint8_t* k0 = J.keys + J.e_koff[0];
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t* k = J.keys + J.e_koff[e];
    const uint32_t kl = J.e_klen[e];  // >= 8: shorter keys failed the decode
    bool bad = false;
    uint64_t p;
    if (L) {
      if (kl - 8 < L) {
        bad = true;
      } else {
        for (uint32_t i = 0; i < L; i++) bad |= k[i] != k0[i];
      }
      p = user_prefix_after(k, kl, L);
      J.e_pfx[e] = p;  // neighbours recompute theirs from the key bytes
    } else {
      p = J.e_pfx[e];
    }
    if (!bad && e > 0 && !run_first(J, e)) {
      const uint8_t* kp = J.keys + J.e_koff[e - 1];
      const uint32_t klp = J.e_klen[e - 1];
      const uint64_t pp = L ? (klp - 8 < L ? 0 : user_prefix_after(kp, klp, L)) : J.e_pfx[e - 1];
      bad = pp > p || (pp == p && ikey_cmp(kp, klp, k, kl) > 0);
    }
    if (bad) set_error(J.ctr, kErrUnsorted, (uint32_t)e);
  }
}

// A single merge child (no round): the merged order is the input order.
__global__ void k_merge_single(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_entries_in;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    J.m_ids[i] = (uint32_t)i;
    J.m_pfx[i] = J.e_pfx[i];
    J.m_tag[i] = J.e_tag[i];
  }
}

// Round r of `rounds` merges groups of 2^r children pairwise: the output of
// pair p (groups 2p and 2p+1) is cut into tiles of `tile` positions.  Round 0
// reads the decoded entries in input order (ids are positions, prefixes and
// tags are e_pfx / e_tag); later rounds read the previous round's arrays.
// Jobs with fewer children copy through, so that every job of a batch ends
// with its merged order in m_ids / m_pfx / m_tag.
struct MergeRound {
  const uint32_t* src_ids;  // nullptr in round 0
  const uint64_t* src_pfx;
  const uint64_t* src_tag;
  uint32_t* dst_ids;
  uint64_t* dst_pfx;
  uint64_t* dst_tag;
};

__device__ __forceinline__ MergeRound merge_round(const JobDev& J, uint32_t r, uint32_t rounds) {
  const bool odd = ((rounds - r) & 1) != 0;
  MergeRound m;
  m.src_ids = r == 0 ? nullptr : (odd ? J.m_tmp : J.m_ids);
  m.src_pfx = r == 0 ? J.e_pfx : (odd ? J.m_pfx_tmp : J.m_pfx);
  m.src_tag = r == 0 ? J.e_tag : (odd ? J.m_tag_tmp : J.m_tag);
  m.dst_ids = odd ? J.m_ids : J.m_tmp;
  m.dst_pfx = odd ? J.m_pfx : J.m_pfx_tmp;
  m.dst_tag = odd ? J.m_tag : J.m_tag_tmp;
  return m;
}

// Pair and tile of the job's g-th merge tile in round r; false past the last.
struct MergeTile {
  uint64_t a0, na, nb;  // the pair's first group [a0, a0 + na), second [a0 + na, + nb)
  uint64_t d0, d1;      // the tile's output positions within the pair
  bool last;            // last tile of its pair
};

__device__ __forceinline__ bool merge_tile(const JobDev& J, uint32_t r, uint64_t g, uint32_t tile,
                                           MergeTile* t) {
  const uint32_t width = 1u << r;
  uint64_t acc = 0;
  for (uint32_t r0 = 0; r0 < J.n_runs; r0 += 2 * width) {
    const uint32_t r1 = min(r0 + width, J.n_runs), r2 = min(r0 + 2 * width, J.n_runs);
    const uint64_t a0 = J.run_entry_begin[r0], b0 = J.run_entry_begin[r1],
                   b1 = J.run_entry_begin[r2];
    const uint64_t len = b1 - a0, tiles = (len + tile - 1) / tile;
    if (g < acc + tiles) {
      const uint64_t k = g - acc;
      t->a0 = a0;
      t->na = b0 - a0;
      t->nb = b1 - b0;
      t->d0 = k * tile;
      t->d1 = min(len, t->d0 + tile);
      t->last = k + 1 == tiles;
      return true;
    }
    acc += tiles;
  }
  return false;
}

__device__ __forceinline__ uint32_t src_id(const MergeRound& m, uint64_t i) {
  return m.src_ids ? m.src_ids[i] : (uint32_t)i;
}

// m_split[g]: elements of the pair's first group before tile g's first
// diagonal (merge path: the first group wins ties, which keeps the children's
// order for equal internal keys, as MergingIterator does).  One thread per
// tile.
__global__ void k_merge_partition(const JobDev* __restrict__ jobs, uint32_t r, uint32_t rounds,
                                  uint32_t tile) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const MergeRound m = merge_round(J, r, rounds);
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < J.cap_merge_tiles;
       g += (uint64_t)gridDim.x * blockDim.x) {
    MergeTile t;
    if (!merge_tile(J, r, g, tile, &t)) break;
    const uint64_t d = t.d0, a = t.a0, b = t.a0 + t.na;
    uint64_t lo = d > t.nb ? d - t.nb : 0, hi = d < t.na ? d : t.na;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      const uint64_t ia = a + mid, ib = b + (d - 1 - mid);
      if (entry_le(J, src_id(m, ia), m.src_pfx[ia], src_id(m, ib), m.src_pfx[ib])) lo = mid + 1;
      else hi = mid;
    }
    J.m_split[g] = (uint32_t)lo;
  }
}

// One tile per CTA step: the tile's stretches of both groups (ids and
// prefixes) are loaded into shared memory with coalesced reads, every thread
// finds its own diagonal there and merges `items` outputs, and the tile is
// written back with coalesced stores; the tags follow by source position
// (two ascending streams).  Only equal prefixes read key bytes.
__global__ void __launch_bounds__(1024) k_merge_tile(const JobDev* __restrict__ jobs, uint32_t r,
                                                     uint32_t rounds, uint32_t items) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  const uint32_t tile = blockDim.x * items;
  extern __shared__ __align__(16) uint8_t merge_smem[];
  uint64_t* in_pfx = reinterpret_cast<uint64_t*>(merge_smem);
  uint64_t* out_pfx = in_pfx + tile;
  uint32_t* in_ids = reinterpret_cast<uint32_t*>(out_pfx + tile);
  uint32_t* out_ids = in_ids + tile;
  uint32_t* out_src = out_ids + tile;  // source position (in the tile) of each output
  const MergeRound m = merge_round(J, r, rounds);
  for (uint64_t g = blockIdx.x; g < J.cap_merge_tiles; g += gridDim.x) {
    MergeTile t;
    if (!merge_tile(J, r, g, tile, &t)) break;
    const uint64_t i0 = J.m_split[g];
    const uint64_t i1 = t.last ? t.na : J.m_split[g + 1];
    if (i1 < i0 || i1 - i0 > t.d1 - t.d0) {
      // cuts out of order: only children out of order give these, and the
      // order check fails such a job first; the tile is skipped, never read
      if (threadIdx.x == 0) set_error(J.ctr, kErrUnsorted, (uint32_t)g);
      continue;
    }
    const uint64_t j0 = t.d0 - i0, j1 = t.d1 - i1;
    const uint32_t na = (uint32_t)(i1 - i0), nb = (uint32_t)(j1 - j0), len = na + nb;
    __syncthreads();  // the previous tile's stores have read the buffers
    for (uint32_t x = threadIdx.x; x < len; x += blockDim.x) {
      const uint64_t i = x < na ? t.a0 + i0 + x : t.a0 + t.na + j0 + (x - na);
      in_ids[x] = src_id(m, i);
      in_pfx[x] = m.src_pfx[i];
    }
    __syncthreads();
    const uint32_t k = threadIdx.x * items;
    if (k < len) {
      // this thread's diagonal within the tile
      uint32_t lo = k > nb ? k - nb : 0, hi = k < na ? k : na;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t jb = na + (k - 1 - mid);
        if (entry_le(J, in_ids[mid], in_pfx[mid], in_ids[jb], in_pfx[jb])) lo = mid + 1;
        else hi = mid;
      }
      uint32_t i = lo, j = k - lo;
      const uint32_t stop = min(len, k + items);
      for (uint32_t o = k; o < stop; o++) {
        const bool take_a =
            i < na && (j >= nb || entry_le(J, in_ids[i], in_pfx[i], in_ids[na + j], in_pfx[na + j]));
        const uint32_t x = take_a ? i++ : na + j++;
        out_ids[o] = in_ids[x];
        out_pfx[o] = in_pfx[x];
        out_src[o] = x;
      }
    }
    __syncthreads();
    const uint64_t o0 = t.a0 + t.d0;
    for (uint32_t x = threadIdx.x; x < len; x += blockDim.x) {
      m.dst_ids[o0 + x] = out_ids[x];
      m.dst_pfx[o0 + x] = out_pfx[x];
      const uint32_t y = out_src[x];
      m.dst_tag[o0 + x] = m.src_tag[y < na ? t.a0 + i0 + y : t.a0 + t.na + j0 + (y - na)];
    }
  }
}

__device__ __forceinline__ bool is_base_level(const JobDev& J, const uint8_t* ukey, uint32_t ulen) {
  for (uint32_t l = 0; l < J.n_base_levels; l++) {
    uint32_t lo = J.base_level_begin[l], hi = J.base_level_begin[l + 1];
    const uint32_t end = hi;
    // first file whose largest user key >= ukey
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (bytes_cmp(ukey, ulen, J.base_keys + J.base_large_off[mid], J.base_large_len[mid]) > 0)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < end &&
        bytes_cmp(ukey, ulen, J.base_keys + J.base_small_off[lo], J.base_small_len[lo]) >= 0)
      return false;
  }
  return true;
}

__device__ __forceinline__ void drop_one(const JobDev& J, const uint32_t* __restrict__ ids,
                                         const uint64_t* __restrict__ pfx,
                                         const uint64_t* __restrict__ tags, uint64_t p) {
  const uint32_t id = ids[p];
  const uint64_t upfx = pfx[p];
  const uint64_t tag = tags[p];
  const uint32_t type = (uint32_t)(tag & 0xff);
  const uint64_t seq = tag >> 8;
  bool drop = false;
  if (type <= 1) {
    bool first = true;
    uint64_t pseq = 0;
    if (p > 0) {
      const uint64_t ptag = tags[p - 1];
      if ((ptag & 0xff) <= 1 && same_user_key(J, ids[p - 1], pfx[p - 1], id, upfx)) {
        first = false;
        pseq = ptag >> 8;
      }
    }
    if (!first && pseq <= J.smallest_snapshot) {
      drop = true;
    } else if (type == 0 && seq <= J.smallest_snapshot &&
               is_base_level(J, J.keys + J.e_koff[id], J.e_klen[id] - 8)) {
      drop = true;
    }
  }
  J.keep[p] = drop ? 0 : 1;
  if (J.n_gp) {
    // grandparents passed: count of g with key > largest[g] (internal-key
    // order); the user-key prefixes decide unless equal
    uint32_t lo = 0, hi = J.n_gp;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      const uint64_t gp = J.gp_upfx[mid];
      const uint32_t mode = J.gp_mode[mid];
      bool after;
      if (mode) {  // the grandparent lies outside the keys' common prefix
        after = mode == 1;
      } else if (gp != upfx) {
        after = upfx > gp;
      } else {
        const uint64_t go = J.gp_key_off[mid];
        const uint32_t gl = (uint32_t)(J.gp_key_off[mid + 1] - go);
        after = ikey_cmp(J.keys + J.e_koff[id], J.e_klen[id], J.gp_keys + go, gl) > 0;
      }
      if (after) lo = mid + 1;
      else hi = mid;
    }
    J.gp_idx[p] = lo;
  }
}

__global__ void k_drop(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint64_t n = J.ctr->n_entries_in;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (uint64_t)gridDim.x * blockDim.x)
    drop_one(J, J.m_ids, J.m_pfx, J.m_tag, p);
}

// gp_first[g] = first merged position whose grandparent count reaches g
// (gp_idx is non-decreasing along the merge order).
__global__ void k_gp_first(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  uint32_t* gp_first = J.gp_first;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > J.n_gp) return;
  const uint64_t n = J.ctr->n_entries_in;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (J.gp_idx[mid] >= g) hi = mid;
    else lo = mid + 1;
  }
  gp_first[g] = (uint32_t)lo;
}

// The cut positions: after a cut at t (or from the first key), the next cut
// is the first key whose running overlap exceeds the limit, i.e. the first
// position whose grandparent count reaches the smallest g with
// prefix[g] - prefix[gp_idx[t]] > limit.  Few cuts; one thread walks them
// over shared-memory copies of the prefix and first-position arrays.
__global__ void k_triggers(const JobDev* __restrict__ jobs, bool in_smem) {
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error;
  __syncthreads();
  if (s_failed) return;
  const uint32_t* gp_first = J.gp_first;
  extern __shared__ uint64_t s_tr[];
  const uint64_t n = J.ctr->n_entries_in;
  const uint32_t G = J.n_gp;
  const uint64_t* pre = J.gp_prefix;
  const uint32_t* first = gp_first;
  if (in_smem) {  // G + 1 prefixes, then G + 1 first positions
    uint32_t* s_first = reinterpret_cast<uint32_t*>(s_tr + G + 1);
    for (uint32_t g = threadIdx.x; g <= G; g += blockDim.x) {
      s_tr[g] = J.gp_prefix[g];
      s_first[g] = gp_first[g];
    }
    pre = s_tr;
    first = s_first;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  uint32_t cnt = 0;
  if (n > 0 && G > 0) {
    const uint64_t limit = (uint64_t)J.max_gp_overlap;
    uint32_t gb = J.gp_idx[0];
    while (true) {
      const uint64_t target = pre[gb] + limit;  // need prefix > target
      uint32_t lo = gb + 1, hi = G + 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pre[mid] > target) hi = mid;
        else lo = mid + 1;
      }
      if (lo > G) break;
      const uint64_t t = first[lo];
      if (t >= n) break;
      if (cnt >= J.cap_triggers) {
        set_error(J.ctr, kErrLimit, 1);
        break;
      }
      J.triggers[cnt++] = (uint32_t)t;
      gb = J.gp_idx[t];
    }
  }
  J.ctr->n_triggers = cnt;
}

__global__ void k_kept_compact(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint32_t* __restrict__ ids = J.m_ids;
  const uint64_t n = J.ctr->n_entries_in;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (uint64_t)gridDim.x * blockDim.x) {
    if (J.keep[p]) {
      const uint32_t k = J.kept_pos[p];
      const uint32_t id = ids[p];
      J.k_koff[k] = J.e_koff[id];
      J.k_klen[k] = J.e_klen[id];
      J.k_voff[k] = J.e_voff[id];
      J.k_vlen[k] = J.e_vlen[id];
      J.k_forced[k] = 0;
    }
  }
}

__global__ void k_forced(const JobDev* __restrict__ jobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nk = J.kept_pos[J.ctr->n_entries_in];
  if (i == 0 && nk > 0) J.k_forced[0] = 1;
  if (i < J.ctr->n_triggers) {
    const uint32_t kp = J.kept_pos[J.triggers[i]];
    if (kp < nk) J.k_forced[kp] = 1;
    J.t_kept[i] = kp;
  }
}

}  // namespace

static unsigned flat_ctas(const Batch& bt, uint64_t items, unsigned per) {
  const uint64_t cap = std::max<uint64_t>(1, bt.ctas_per_job ? bt.ctas_per_job : 148 * 8 / bt.B);
  return grid_x(items, per, cap);
}

// Merge tile (threads x items, at most kMergeMaxTile) and the shared memory
// it takes: ids and prefixes of the tile's input and output and each output's
// source position.
static uint32_t merge_items_of(const Batch& bt) {
  uint32_t items = std::max<uint32_t>(1, bt.merge_items);
  while ((uint64_t)bt.merge_threads * items > kMergeMaxTile && items > 1) items >>= 1;
  return items;
}

void merge_kernel_attributes() {
  cudaFuncSetAttribute(k_merge_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(kMergeSmemPerPos * kMergeMaxTile));
}

uint64_t merge_tile_capacity(uint64_t entries, uint32_t runs) {
  // tiles of at least 64 positions, one partial tile per pair
  return entries / 64 + runs + 2;
}

void launch_key_skip(const Batch& bt, cudaStream_t st) {
  note_launch(), k_key_skip<<<dim3(1, bt.B), 256, 0, st>>>(bt.d);
  note_launch(), k_prefix<<<dim3(flat_ctas(bt, bt.max_entries, 256), bt.B), 256, 0, st>>>(bt.d);
}

void launch_merge(const Batch& bt, cudaStream_t st) {
  if (bt.merge_rounds == 0) {
    note_launch(), k_merge_single<<<dim3(flat_ctas(bt, bt.max_entries, 256), bt.B), 256, 0, st>>>(
        bt.d);
    return;
  }
  const uint32_t items = merge_items_of(bt);
  const uint32_t threads = bt.merge_threads;
  const uint32_t tile = threads * items;
  const uint64_t tiles = bt.max_entries / tile + bt.max_runs + 1;
  for (uint32_t r = 0; r < bt.merge_rounds; r++) {
    note_launch(), k_merge_partition<<<dim3(grid_x(tiles, 128, 148 * 16), bt.B), 128, 0, st>>>(
        bt.d, r, bt.merge_rounds, tile);
    note_launch(), k_merge_tile<<<dim3(flat_ctas(bt, tiles, 1), bt.B), threads,
                                  kMergeSmemPerPos * (size_t)tile, st>>>(bt.d, r, bt.merge_rounds,
                                                                         items);
  }
}

void launch_drop(const Batch& bt, cudaStream_t st) {
  note_launch(), k_drop<<<dim3(flat_ctas(bt, bt.max_entries, 256), bt.B), 256, 0, st>>>(bt.d);
}

void launch_triggers(const Batch& bt, cudaStream_t st) {
  if (bt.max_gp)
    note_launch(), k_gp_first<<<dim3((bt.max_gp + 1 + 255) / 256, bt.B), 256, 0, st>>>(bt.d);
  const size_t smem = (size_t)(bt.max_gp + 1) * 12;
  const bool in_smem = smem + 64 <= 48 * 1024;  // with the kernel's static shared memory
  note_launch(), k_triggers<<<dim3(1, bt.B), 256, in_smem ? smem : 0, st>>>(bt.d, in_smem);
}

void launch_kept_compact(const Batch& bt, cudaStream_t st) {
  note_launch(), k_kept_compact<<<dim3(flat_ctas(bt, bt.max_entries, 256), bt.B), 256, 0, st>>>(bt.d);
  note_launch(), k_forced<<<dim3((bt.max_cap_triggers + 255) / 256 + 1, bt.B), 256, 0, st>>>(bt.d);
}

}  // namespace lc
