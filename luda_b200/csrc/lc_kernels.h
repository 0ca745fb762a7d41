// Host-callable launchers for the engine's kernels.  Each launcher enqueues
// work on `st` and never synchronises; counts that are only known on the
// device are read by the kernels from JobDev::ctr, and grids are sized from
// host-side capacities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lc_job.h"

namespace lc {

// Kernel launches made by the calling thread (each job runs on one thread).
void note_launch(uint32_t n = 1);
uint32_t launches_on_this_thread();

// lc_scan.cu
template <typename TI, typename TO>
void scan_exclusive(const TI* in, TO* out, const uint64_t* n_dev, uint64_t n_cap, TO* scratch,
                    uint64_t* total_out, cudaStream_t st);
uint64_t scan_scratch_elems(uint64_t n_cap);

// lc_crc.cu -- masked CRC32C of one buffer; `counter` must be zero at launch
void launch_crc32c_chunks(const uint8_t* data, uint64_t n, uint32_t* partials, uint32_t* counter,
                          uint32_t* out, cudaStream_t st);

// lc_decode.cu -- input tables -> decoded entries
void launch_table_index_count(const JobDev& J, cudaStream_t st);
void launch_table_index_entries(const JobDev& J, cudaStream_t st);
void launch_block_count(const JobDev& J, uint64_t n_blocks_cap, cudaStream_t st);
void launch_run_bounds(const JobDev& J, cudaStream_t st);
void launch_block_decode(const JobDev& J, uint64_t n_blocks_cap, cudaStream_t st);
void launch_entries_from_offsets(const JobDev& J, const uint64_t* koffs, const uint64_t* voffs,
                                 uint64_t n, cudaStream_t st);

// lc_merge.cu -- merge, drop rule, grandparent cuts, survivors
void launch_iota(uint32_t* ids, uint64_t n, cudaStream_t st);
void launch_merge_round(const JobDev& J, const uint32_t* src, uint32_t* dst, uint32_t width,
                        uint64_t n, cudaStream_t st);
void launch_drop(const JobDev& J, uint64_t n, cudaStream_t st);
void launch_triggers(const JobDev& J, uint64_t n, uint32_t* gp_first, cudaStream_t st);
void launch_kept_compact(const JobDev& J, uint64_t n, cudaStream_t st);

// lc_encode.cu -- survivors -> output tables
void launch_sizes(const JobDev& J, uint64_t n_cap, cudaStream_t st);
void launch_next(const JobDev& J, uint64_t n_cap, cudaStream_t st);
void launch_chain(const JobDev& J, uint64_t n_cap, cudaStream_t st);
void launch_block_list(const JobDev& J, uint64_t n_cap, cudaStream_t st);
void launch_block_sizes(const JobDev& J, uint32_t* tmp32, uint64_t nb_cap, cudaStream_t st);
void launch_files(const JobDev& J, uint64_t nb_cap, cudaStream_t st);
void launch_block_layout(const JobDev& J, uint64_t nb_cap, cudaStream_t st);
void launch_file_layout(const JobDev& J, cudaStream_t st);
void launch_encode_blocks(const JobDev& J, uint64_t nb, cudaStream_t st);
void launch_encode_rest(const JobDev& J, uint64_t nb, uint32_t n_files, cudaStream_t st);
void launch_file_keys(const JobDev& J, uint32_t cap_files, uint8_t* key_out, uint64_t* key_off,
                      cudaStream_t st);

}  // namespace lc
