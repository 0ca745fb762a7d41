// Allocation-free masked CRC32C: lc_crc32c_noalloc (include/luda_b200.h).
//
// Same computation as lc_crc32c (chunk registers combined by the last CTA,
// lc_crc_chunks.cuh), but the scratch lives in a fixed file-scope device
// array instead of the engine's memory pool, so the call allocates nothing.
// The array is part of the loaded module: every device that loads this
// library holds it (kNoAllocCrcMaxChunks + 1 words, about 64 KiB) until the
// process exits.
//
// Host code must not use the array's name as a device address (in host code
// it is only a stand-in), so the first call on each device looks the address
// up with cudaGetSymbolAddress while that device is current and caches it.
// The cached address belongs to the device's current context: after a
// cudaDeviceReset the module is loaded again, possibly elsewhere, so the
// entry point must not be used across a device reset.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/luda_b200.h"
#include "lc_crc_chunks.cuh"
#include "lc_kernels.h"

namespace {

// Largest buffer: kNoAllocCrcMaxChunks chunks of kCrcChunkBytes = 1 GiB.
constexpr uint32_t kNoAllocCrcMaxChunks = 16384;
constexpr uint64_t kNoAllocCrcMaxBytes = (uint64_t)kNoAllocCrcMaxChunks * lc::kCrcChunkBytes;
constexpr int kMaxDevices = 64;

// [0, kNoAllocCrcMaxChunks): per-chunk CRC registers; [kNoAllocCrcMaxChunks]:
// the ticket counter, cleared before every launch.
__device__ __align__(256) uint32_t g_noalloc_crc_scratch[kNoAllocCrcMaxChunks + 1];

std::mutex g_setup_mu;
uint32_t* g_scratch_addr[kMaxDevices] = {};

__global__ void __launch_bounds__(lc::kCrcChunkThreads)
    k_crc32c_chunks_static(const uint8_t* data, uint64_t n, uint32_t* scratch, uint32_t* out) {
  lc::crc32c_chunks_body(data, n, scratch, scratch + kNoAllocCrcMaxChunks, out);
}

// Records the failing step (and the CUDA error, if any) as the calling
// thread's lc_last_error() text, like the other entry points, and returns s.
inline lc_status noalloc_fail(lc_status s, const char* what, cudaError_t e = cudaSuccess) {
  std::string m(what);
  if (e != cudaSuccess) m += std::string(": ") + cudaGetErrorString(e);
  lc::set_last_error(m);
  return s;
}

}  // namespace

extern "C" {

lc_status lc_crc32c_noalloc(const uint8_t* d_data, uint64_t n, uint32_t* d_masked_crc,
                            void* stream) {
  if (!d_masked_crc || (n && !d_data))
    return noalloc_fail(LC_ERR_INVALID_ARG, "lc_crc32c_noalloc: null device pointer");
  if (n > kNoAllocCrcMaxBytes)
    return noalloc_fail(LC_ERR_UNSUPPORTED,
                        "lc_crc32c_noalloc: buffer larger than the 1 GiB static scratch limit");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(LC_ERR_CUDA, "lc_crc32c_noalloc: cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(LC_ERR_UNSUPPORTED, "lc_crc32c_noalloc: device ordinal beyond 63");
  uint32_t* scratch;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> g(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_crc_scratch);
      if (e != cudaSuccess)
        return noalloc_fail(LC_ERR_CUDA, "lc_crc32c_noalloc: cudaGetSymbolAddress", e);
      g_scratch_addr[dev] = (uint32_t*)p;
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  // the ticket counter must start at zero; the registers are overwritten
  e = cudaMemsetAsync(scratch + kNoAllocCrcMaxChunks, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return noalloc_fail(LC_ERR_CUDA, "lc_crc32c_noalloc: clear counter", e);
  k_crc32c_chunks_static<<<lc::crc32c_chunk_count(n), lc::kCrcChunkThreads, 0, st>>>(
      d_data, n, scratch, d_masked_crc);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LC_ERR_CUDA, "lc_crc32c_noalloc: launch", e);
  return LC_OK;
}

}  // extern "C"
