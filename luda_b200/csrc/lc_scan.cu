// Device-wide exclusive prefix sums (reduce, scan of tile sums, scan).
//
// The element count may live in device memory (n_dev) so that a scan can be
// enqueued before the producing kernel's count is known on the host; the grid
// is sized from a host-side capacity and tiles past the count exit early.
// out has n+1 entries: out[n] is the total.
#include <cuda_runtime.h>
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
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* total) {
  __shared__ T warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  T incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nwarps ? warp_sums[lane] : T(0);
    T wi = warp_incl_scan(w);
    if (lane < nwarps) warp_sums[lane] = wi - w;
    if (lane == nwarps - 1) warp_sums[31] = wi;
  }
  __syncthreads();
  T res = warp_sums[warp] + incl - v;
  *total = warp_sums[31];
  __syncthreads();
  return res;
}

__device__ __forceinline__ uint64_t resolve_n(const uint64_t* n_dev, uint64_t n_host) {
  return n_dev ? *n_dev : n_host;
}

template <typename TI, typename TO>
__global__ void k_tile_reduce(const TI* in, const uint64_t* n_dev, uint64_t n_host,
                              TO* tile_sums) {
  const uint64_t n = resolve_n(n_dev, n_host);
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  TO s = 0;
  if (base < n) {
    for (int k = 0; k < kScanItems; k++) {
      uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
      if (i < n) s += (TO)in[i];
    }
  }
  TO total;
  block_excl_scan<TO>(s, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <typename TO>
__global__ void k_scan_tiles(TO* tile_sums, uint32_t n_tiles) {
  TO carry = 0;
  for (uint32_t base = 0; base < n_tiles; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    TO v = i < n_tiles ? tile_sums[i] : TO(0);
    TO total;
    TO ex = block_excl_scan<TO>(v, &total);
    if (i < n_tiles) tile_sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) tile_sums[n_tiles] = carry;
}

template <typename TI, typename TO>
__global__ void k_tile_scan(const TI* in, const uint64_t* n_dev, uint64_t n_host,
                            const TO* tile_offsets, TO* out, uint64_t* total_out) {
  const uint64_t n = resolve_n(n_dev, n_host);
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  if (base > n) return;
  TO vals[kScanItems];
  TO s = 0;
  const uint64_t tb = base + (uint64_t)threadIdx.x * kScanItems;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t i = tb + k;
    vals[k] = i < n ? (TO)in[i] : TO(0);
    s += vals[k];
  }
  TO total;
  TO ex = block_excl_scan<TO>(s, &total) + tile_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t i = tb + k;
    if (i < n) out[i] = ex;
    else if (i == n) {
      out[n] = ex;
      if (total_out) *total_out = (uint64_t)ex;
    }
    ex += vals[k];
  }
}

}  // namespace

template <typename TI, typename TO>
void scan_exclusive(const TI* in, TO* out, const uint64_t* n_dev, uint64_t n_cap,
                    TO* scratch, uint64_t* total_out, cudaStream_t st) {
  uint32_t tiles = (uint32_t)((n_cap + 1 + kTile - 1) / kTile);
  if (tiles == 0) tiles = 1;
  note_launch(3);
  k_tile_reduce<TI, TO><<<tiles, kScanThreads, 0, st>>>(in, n_dev, n_cap, scratch);
  k_scan_tiles<TO><<<1, 1024, 0, st>>>(scratch, tiles);
  k_tile_scan<TI, TO><<<tiles, kScanThreads, 0, st>>>(in, n_dev, n_cap, scratch, out, total_out);
}

uint64_t scan_scratch_elems(uint64_t n_cap) { return (n_cap + 1 + kTile - 1) / kTile + 2; }

template void scan_exclusive<uint32_t, uint64_t>(const uint32_t*, uint64_t*, const uint64_t*,
                                                 uint64_t, uint64_t*, uint64_t*, cudaStream_t);
template void scan_exclusive<uint64_t, uint64_t>(const uint64_t*, uint64_t*, const uint64_t*,
                                                 uint64_t, uint64_t*, uint64_t*, cudaStream_t);
template void scan_exclusive<uint8_t, uint32_t>(const uint8_t*, uint32_t*, const uint64_t*,
                                                uint64_t, uint32_t*, uint64_t*, cudaStream_t);
template void scan_exclusive<uint32_t, uint32_t>(const uint32_t*, uint32_t*, const uint64_t*,
                                                 uint64_t, uint32_t*, uint64_t*, cudaStream_t);

}  // namespace lc
