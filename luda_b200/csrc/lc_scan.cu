// Exclusive prefix sums of per-job arrays in two launches for a whole batch
// (grid y = job): per-tile sums, then the scan of each tile from its offset,
// which every CTA sums from the tile sums before it.
//
// The array and its length are chosen by a selector from the job descriptor;
// the length lives in device memory, so a scan can be enqueued before the
// producing kernel's count is known on the host.  The grid is sized from a
// host-side capacity and tiles past the count exit early.  out has n+1
// entries: out[n] is the total, optionally also stored to a counter.
#include <cuda_runtime.h>
#include <algorithm>
#include <stdint.h>

#include "lc_kernels.h"

namespace lc {

namespace {
thread_local uint32_t t_launches = 0;
}  // namespace

void note_launch(uint32_t n) { t_launches += n; }
uint32_t launches_on_this_thread() { return t_launches; }

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kTile = kScanThreads * kScanItems;

template <int S>
struct ScanOf;
template <>
struct ScanOf<kScanTblBlocks> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.tbl_nblocks; }
  static __device__ TO* out(const JobDev& J) { return J.tbl_block_base; }
  static __device__ uint64_t n(const JobDev& J) { return J.n_tables; }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->n_blocks_in; }
};
template <>
struct ScanOf<kScanBlkEnt> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.blk_nent; }
  static __device__ TO* out(const JobDev& J) { return J.blk_ent_base; }
  static __device__ uint64_t n(const JobDev& J) { return min(J.ctr->n_blocks_in, J.cap_blocks_in); }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->n_entries_in; }
};
template <>
struct ScanOf<kScanBlkKey> {
  using TI = uint64_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.blk_kbytes; }
  static __device__ TO* out(const JobDev& J) { return J.blk_key_base; }
  static __device__ uint64_t n(const JobDev& J) { return min(J.ctr->n_blocks_in, J.cap_blocks_in); }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->key_bytes_in; }
};
template <>
struct ScanOf<kScanKeep> {
  using TI = uint8_t;
  using TO = uint32_t;
  static __device__ const TI* in(const JobDev& J) { return J.keep; }
  static __device__ TO* out(const JobDev& J) { return J.kept_pos; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_entries_in; }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->n_kept; }
};
template <>
struct ScanOf<kScanBstart> {
  using TI = uint8_t;
  using TO = uint32_t;
  static __device__ const TI* in(const JobDev& J) { return J.k_bstart; }
  static __device__ TO* out(const JobDev& J) { return J.k_block; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_kept; }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->n_blocks_out; }
};
template <>
struct ScanOf<kScanBcum> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.tmp32; }
  static __device__ TO* out(const JobDev& J) { return J.b_cum; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_blocks_out; }
  static __device__ uint64_t* total(const JobDev&) { return nullptr; }
};
template <>
struct ScanOf<kScanGcum> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.b_gbytes; }
  static __device__ TO* out(const JobDev& J) { return J.b_gcum; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_blocks_out; }
  static __device__ uint64_t* total(const JobDev&) { return nullptr; }
};
template <>
struct ScanOf<kScanIcum> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.b_isize; }
  static __device__ TO* out(const JobDev& J) { return J.b_icum; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_blocks_out; }
  static __device__ uint64_t* total(const JobDev&) { return nullptr; }
};

template <>
struct ScanOf<kScanDecKey> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.k_klen; }
  static __device__ TO* out(const JobDev& J) { return J.dec_kcum; }  // null: job skipped
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_kept; }
  static __device__ uint64_t* total(const JobDev&) { return nullptr; }
};

template <>
struct ScanOf<kScanKb> {
  using TI = uint32_t;
  using TO = uint64_t;
  static __device__ const TI* in(const JobDev& J) { return J.k_b; }
  static __device__ TO* out(const JobDev& J) { return J.k_pb; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_kept; }
  static __device__ uint64_t* total(const JobDev&) { return nullptr; }
};

template <>
struct ScanOf<kScanDecKlen> {
  using TI = uint32_t;
  using TO = uint32_t;
  static __device__ const TI* in(const JobDev& J) { return J.e_klen; }
  static __device__ TO* out(const JobDev& J) { return J.e_koff; }
  static __device__ uint64_t n(const JobDev& J) { return J.ctr->n_entries_in; }
  static __device__ uint64_t* total(const JobDev& J) { return &J.ctr->key_cursor; }
};

// Tile-sum scratch of a scan (the scans of a job run one after another).
template <int S>
__device__ __forceinline__ uint64_t* scan_tiles_of(const JobDev& J) {
  return J.scan_scratch;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Exclusive scan across the CTA; returns the exclusive prefix, *total = sum.
// The total has its own slot: with 32 warps every one of warp_sums[0..31]
// holds a warp's exclusive prefix.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* total) {
  __shared__ T warp_sums[33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  T incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nwarps ? warp_sums[lane] : T(0);
    T wi = warp_incl_scan(w);
    if (lane < nwarps) warp_sums[lane] = wi - w;
    if (lane == 31) warp_sums[32] = wi;  // lanes past nwarps add nothing
  }
  __syncthreads();
  T res = warp_sums[warp] + incl - v;
  *total = warp_sums[32];
  __syncthreads();
  return res;
}

template <int S>
__global__ void k_tile_reduce(const JobDev* __restrict__ jobs) {
  using SP = ScanOf<S>;
  using TO = typename SP::TO;
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error || SP::out(J) == nullptr;
  __syncthreads();
  if (s_failed) return;
  const uint64_t n = SP::n(J);
  TO* tile_sums = reinterpret_cast<TO*>(scan_tiles_of<S>(J));
  const typename SP::TI* in = SP::in(J);
  for (uint64_t t = blockIdx.x; t * kTile <= n; t += gridDim.x) {
    const uint64_t base = t * kTile;
    TO s = 0;
    for (int k = 0; k < kScanItems; k++) {
      const uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
      if (i < n) s += (TO)in[i];
    }
    TO total;
    block_excl_scan<TO>(s, &total);
    if (threadIdx.x == 0) tile_sums[t] = total;
  }
}

// Sum of a[lo, hi) over the CTA (every thread gets it).
template <typename T>
__device__ __forceinline__ T block_sum(const T* a, uint64_t lo, uint64_t hi) {
  T v = 0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) v += a[i];
  T total;
  block_excl_scan<T>(v, &total);
  return total;
}

template <int S>
__global__ void k_tile_scan(const JobDev* __restrict__ jobs) {
  using SP = ScanOf<S>;
  using TO = typename SP::TO;
  const JobDev& J = jobs[blockIdx.y];
  __shared__ uint32_t s_failed;  // read once per CTA: the CTA's barriers stay uniform
  if (threadIdx.x == 0) s_failed = J.ctr->error || SP::out(J) == nullptr;
  __syncthreads();
  if (s_failed) return;
  const uint64_t n = SP::n(J);
  const TO* tile_sums = reinterpret_cast<const TO*>(scan_tiles_of<S>(J));
  const uint64_t n_tiles = n / kTile + 1;
  const typename SP::TI* in = SP::in(J);
  TO* out = SP::out(J);
  uint64_t* total_out = SP::total(J);
  // offset of this CTA's first tile: the sums of the tiles before it; each
  // step of the grid stride adds the sums of the tiles it skips
  TO carry = block_sum<TO>(tile_sums, 0, (uint64_t)blockIdx.x < n_tiles ? blockIdx.x : n_tiles);
  for (uint64_t t = blockIdx.x; t * kTile <= n; t += gridDim.x) {
    const uint64_t base = t * kTile;
    TO vals[kScanItems];
    TO s = 0;
    const uint64_t tb = base + (uint64_t)threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      const uint64_t i = tb + k;
      vals[k] = i < n ? (TO)in[i] : TO(0);
      s += vals[k];
    }
    TO total;
    TO ex = block_excl_scan<TO>(s, &total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      const uint64_t i = tb + k;
      if (i < n) {
        out[i] = ex;
      } else if (i == n) {
        out[n] = ex;
        if (total_out) *total_out = (uint64_t)ex;
      }
      ex += vals[k];
    }
    if ((t + gridDim.x) * kTile <= n)  // another tile of this CTA follows
      carry += block_sum<TO>(tile_sums, t, t + gridDim.x < n_tiles ? t + gridDim.x : n_tiles);
  }
}

template <int S>
void scan_sel(const Batch& bt, uint64_t n_cap, cudaStream_t st) {
  const unsigned tiles = grid_x(n_cap + 1, kTile, 148 * 8);
  // one tile (n + 1 <= kTile for every job of the batch): no tile sums to
  // add, so the scan pass alone does it
  const bool one_tile = n_cap + 1 <= kTile;
  note_launch(one_tile ? 1 : 2);
  if (!one_tile) k_tile_reduce<S><<<dim3(tiles, bt.B), kScanThreads, 0, st>>>(bt.d);
  k_tile_scan<S><<<dim3(tiles, bt.B), kScanThreads, 0, st>>>(bt.d);
}

}  // namespace

void scan_batch(ScanSel sel, const Batch& bt, uint64_t n_cap, cudaStream_t st) {
  switch (sel) {
    case kScanTblBlocks: scan_sel<kScanTblBlocks>(bt, n_cap, st); break;
    case kScanBlkEnt: scan_sel<kScanBlkEnt>(bt, n_cap, st); break;
    case kScanBlkKey: scan_sel<kScanBlkKey>(bt, n_cap, st); break;
    case kScanKeep: scan_sel<kScanKeep>(bt, n_cap, st); break;
    case kScanBstart: scan_sel<kScanBstart>(bt, n_cap, st); break;
    case kScanBcum: scan_sel<kScanBcum>(bt, n_cap, st); break;
    case kScanGcum: scan_sel<kScanGcum>(bt, n_cap, st); break;
    case kScanIcum: scan_sel<kScanIcum>(bt, n_cap, st); break;
    case kScanDecKey: scan_sel<kScanDecKey>(bt, n_cap, st); break;
    case kScanKb: scan_sel<kScanKb>(bt, n_cap, st); break;
    case kScanDecKlen: scan_sel<kScanDecKlen>(bt, n_cap, st); break;
  }
}

// tile sums for arrays of up to n_cap elements (TO up to 8 bytes)
uint64_t scan_scratch_elems(uint64_t n_cap) { return (n_cap + 1) / kTile + 2; }

namespace {

// Small control transfers (descriptors, counters, per-file results) between
// device memory and mapped pinned host memory, done by SM loads and stores
// over PCIe rather than by a copy engine.  A copy engine serves the streams'
// copies in turn, so with other jobs' bulk uploads and downloads in flight a
// few-KB cudaMemcpyAsync waited behind megabytes of them and held up its
// job's next kernels.  16-byte words, then the last bytes.
__global__ void k_xfer(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, uint64_t n) {
  const uint64_t n16 = n / 16;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (uint64_t i = t; i < n16; i += stride)
    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
  for (uint64_t i = n16 * 16 + t; i < n; i += stride) dst[i] = src[i];
}

}  // namespace

bool launch_xfer(void* dst, const void* src, uint64_t n, cudaStream_t st) {
  if (((uintptr_t)dst | (uintptr_t)src) & 15) return false;
  if (!n) return true;
  const uint64_t words = n / 16 + 1;
  const unsigned grid = (unsigned)std::min<uint64_t>((words + 255) / 256, 148);
  note_launch(1);
  k_xfer<<<grid, 256, 0, st>>>((uint8_t*)dst, (const uint8_t*)src, n);
  return true;
}

}  // namespace lc
