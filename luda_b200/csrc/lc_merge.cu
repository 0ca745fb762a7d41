// Merge and drop: decoded runs -> survivors in output order.
//
// * Merge: the reference merges its children with MergingIterator
//   (table/merger.cc:148, linear FindSmallest; on equal keys the earlier child
//   wins).  Here the children are merged pairwise in rounds with merge path:
//   each thread finds its output diagonal by binary search and merges a short
//   stretch.  Ties go to the left (earlier) group, which keeps child order.
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

__global__ void k_iota(const JobDev* __restrict__ jobs, uint32_t rounds) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  uint32_t* ids = (rounds & 1) ? J.m_tmp : J.m_ids;  // the buffer round 0 reads
  const uint64_t n = J.ctr->n_entries_in;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    ids[i] = (uint32_t)i;
}

// Round `r` of `rounds`: groups of width = 2^r merge children; pairs (2p,
// 2p+1) merge.  Jobs with fewer children copy through, so every job of a
// batch ends with its merged order in m_ids.
__global__ void k_merge_round(const JobDev* __restrict__ jobs, uint32_t r, uint32_t rounds,
                              uint32_t items) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.ctr->error) return;  // a failed job does no more work
  const uint32_t* __restrict__ src = ((rounds - r) & 1) ? J.m_tmp : J.m_ids;
  uint32_t* __restrict__ dst = ((rounds - r) & 1) ? J.m_ids : J.m_tmp;
  const uint32_t width = 1u << r;
  const uint64_t n = J.run_entry_begin[J.n_runs];
  for (uint64_t o0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * items; o0 < n;
       o0 += (uint64_t)gridDim.x * blockDim.x * items) {
    const uint64_t o1 = min(n, o0 + items);
    uint64_t o = o0;
    while (o < o1) {
      // find the pair that owns output position o
      const uint32_t pair_runs = 2 * width;
      uint32_t r0 = 0;
      while (true) {
        const uint32_t r2 = min(r0 + pair_runs, J.n_runs);
        if (o < J.run_entry_begin[r2]) break;
        r0 = r2;
      }
      const uint32_t r1 = min(r0 + width, J.n_runs);
      const uint32_t r2 = min(r0 + pair_runs, J.n_runs);
      const uint64_t a0 = J.run_entry_begin[r0], b0 = J.run_entry_begin[r1],
                     b1 = J.run_entry_begin[r2];
      const uint64_t na = b0 - a0, nb = b1 - b0;
      const uint64_t stop = min(o1, b1);
      if (nb == 0) {
        for (; o < stop; o++) dst[o] = src[o];
        continue;
      }
      const uint32_t* A = src + a0;
      const uint32_t* B = src + b0;
      const uint64_t d = o - a0;
      uint64_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (entry_cmp(J, A[mid], B[d - 1 - mid]) <= 0) lo = mid + 1;
        else hi = mid;
      }
      uint64_t i = lo, j = d - lo;
      for (; o < stop; o++) {
        const bool take_a = i < na && (j >= nb || entry_cmp(J, A[i], B[j]) <= 0);
        dst[o] = take_a ? A[i++] : B[j++];
      }
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
                                         uint64_t p) {
  const uint32_t id = ids[p];
  const uint8_t* key = J.keys + J.e_koff[id];
  const uint32_t klen = J.e_klen[id];
  const uint64_t tag = ld_le64(key + klen - 8);
  const uint32_t type = (uint32_t)(tag & 0xff);
  const uint64_t seq = tag >> 8;
  bool drop = false;
  if (type <= 1) {
    bool first = true;
    uint64_t pseq = 0;
    if (p > 0) {
      const uint32_t pid = ids[p - 1];
      const uint8_t* pkey = J.keys + J.e_koff[pid];
      const uint64_t ptag = ld_le64(pkey + J.e_klen[pid] - 8);
      if ((ptag & 0xff) <= 1 && same_user_key(J, pid, id)) {
        first = false;
        pseq = ptag >> 8;
      }
    }
    if (!first && pseq <= J.smallest_snapshot) {
      drop = true;
    } else if (type == 0 && seq <= J.smallest_snapshot && is_base_level(J, key, klen - 8)) {
      drop = true;
    }
  }
  J.keep[p] = drop ? 0 : 1;
  if (J.n_gp) {
    // grandparents passed: count of g with key > largest[g]
    uint32_t lo = 0, hi = J.n_gp;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      const uint64_t go = J.gp_key_off[mid];
      const uint32_t gl = (uint32_t)(J.gp_key_off[mid + 1] - go);
      if (ikey_cmp(key, klen, J.gp_keys + go, gl) > 0) lo = mid + 1;
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
    drop_one(J, J.m_ids, p);
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
      J.k_ids[k] = ids[p];
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
  }
}

}  // namespace

static unsigned flat_ctas(const Batch& bt, uint64_t items, unsigned per) {
  const uint64_t cap = std::max<uint64_t>(1, bt.ctas_per_job ? bt.ctas_per_job : 148 * 8 / bt.B);
  return grid_x(items, per, cap);
}

void launch_merge(const Batch& bt, cudaStream_t st) {
  note_launch(), k_iota<<<dim3(flat_ctas(bt, bt.max_entries, 256), bt.B), 256, 0, st>>>(
      bt.d, bt.merge_rounds);
  const uint32_t items = bt.merge_items;
  const uint32_t threads = bt.merge_threads;
  for (uint32_t r = 0; r < bt.merge_rounds; r++)
    note_launch(), k_merge_round<<<dim3(flat_ctas(bt, (bt.max_entries + items - 1) / items, threads),
                                        bt.B), threads, 0, st>>>(bt.d, r, bt.merge_rounds, items);
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
