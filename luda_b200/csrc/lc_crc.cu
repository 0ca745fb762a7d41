// Chunked masked CRC32C of one buffer (see lc_crc_chunks.cuh), with scratch
// (per-chunk registers and a ticket counter) supplied by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lc_crc_chunks.cuh"
#include "lc_kernels.h"

namespace lc {

namespace {
__global__ void __launch_bounds__(kCrcChunkThreads)
    k_crc32c_chunks(const uint8_t* data, uint64_t n, uint32_t* partials, uint32_t* counter,
                    uint32_t* out) {
  crc32c_chunks_body(data, n, partials, counter, out);
}
}  // namespace

void launch_crc32c_chunks(const uint8_t* data, uint64_t n, uint32_t* partials,
                          uint32_t* counter, uint32_t* out, cudaStream_t st) {
  note_launch();
  k_crc32c_chunks<<<crc32c_chunk_count(n), kCrcChunkThreads, 0, st>>>(data, n, partials, counter,
                                                                        out);
}

}  // namespace lc
