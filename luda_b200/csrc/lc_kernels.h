// Host-callable launchers for the engine's kernels.
//
// Every kernel serves a batch of jobs in one launch: the grid's y dimension is
// the job index, and each kernel reads its job's descriptor from a device
// array (`jobs[blockIdx.y]`).  A plain compaction is a batch of one.  Launchers
// enqueue work on `st` and never synchronise; counts that are only known on
// the device are read by the kernels from each job's Counters, and grids are
// sized from host-side capacities (maxima over the batch).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "lc_job.h"

namespace lc {

// Sets the calling thread's lc_last_error() text.
void set_last_error(const std::string& msg);

// Kernel launches made by the calling thread (each batch runs on one thread).
void note_launch(uint32_t n = 1);
uint32_t launches_on_this_thread();

// Raise the dynamic shared-memory limits of the kernels that need more than
// 48 KiB; once per device, with that device current, before any launch or
// stream capture.
void decode_kernel_attributes();
void encode_kernel_attributes();
void merge_kernel_attributes();

// Chunks per group in the block-chain resolution.
constexpr uint32_t kChainGroup = 64;

// Largest merge tile (threads x items) and the shared memory the tile takes
// per position.
constexpr uint32_t kMergeMaxTile = 4096;
constexpr uint32_t kMergeSmemPerPos = 28;
// Entries of m_split a job needs for `entries` entries in `runs` children.
uint64_t merge_tile_capacity(uint64_t entries, uint32_t runs);

struct Batch {
  const JobDev* d = nullptr;  // device array of B job descriptors
  uint32_t B = 0;
  // maxima over the batch, for grid sizes
  uint32_t max_tables = 0, max_gp = 0, max_cap_triggers = 0, max_cap_files = 0;
  uint64_t max_blocks_in = 0, max_entries = 0;
  uint32_t merge_rounds = 0;
  uint32_t max_runs = 1;
  uint32_t chunk = 4096;
  uint32_t chain_smem_words = 11 * 1024;
  bool any_verify = false;  // some job checks its input blocks' CRCs
  bool any_keep_decoded = false;  // some job keeps its outputs' decoded form
  // tunables (chosen by the autotuner in lc_engine.cu)
  uint32_t ctas_per_job = 0;  // grid x of the grid-stride kernels; 0 = from the sizes
  uint32_t merge_items = 8;   // outputs per thread in a merge round
  uint32_t merge_threads = 256;  // threads per merge CTA (tile = threads * items)
};

// lc_scan.cu -- exclusive prefix sums over per-job arrays chosen by selector
enum ScanSel : int {
  kScanTblBlocks = 0,  // tbl_nblocks -> tbl_block_base      (total: n_blocks_in)
  kScanBlkEnt,         // blk_nent -> blk_ent_base           (total: n_entries_in)
  kScanBlkKey,         // blk_kbytes -> blk_key_base         (total: key_bytes_in)
  kScanKeep,           // keep -> kept_pos                   (total: n_kept)
  kScanBstart,         // k_bstart -> k_block                (total: n_blocks_out)
  kScanBcum,           // tmp32 -> b_cum
  kScanGcum,           // b_gbytes -> b_gcum
  kScanIcum,           // b_isize -> b_icum
  kScanDecKey,         // k_klen -> dec_kcum (jobs that keep their decoded form)
  kScanKb,             // k_b -> k_pb (block size estimates)
  kScanDecKlen,        // e_klen -> e_koff (decode: key places)  (total: key_cursor)
};
void scan_batch(ScanSel sel, const Batch& bt, uint64_t n_cap, cudaStream_t st);
uint64_t scan_scratch_elems(uint64_t n_cap);

// lc_crc.cu -- masked CRC32C of one buffer; `counter` must be zero at launch
void launch_crc32c_chunks(const uint8_t* data, uint64_t n, uint32_t* partials, uint32_t* counter,
                          uint32_t* out, cudaStream_t st);

// lc_decode.cu -- input tables -> decoded entries
void launch_table_index_count(const Batch& bt, cudaStream_t st);
void launch_table_index_entries(const Batch& bt, cudaStream_t st);
void launch_block_count(const Batch& bt, cudaStream_t st);     // exact key counts (full walk)
void launch_block_restarts(const Batch& bt, cudaStream_t st);  // entry counts from restart words
void launch_run_bounds(const Batch& bt, cudaStream_t st);
// Checks the CRC32C trailer of every input data block of the jobs that ask
// for it (verify_checksums), after the block list is known.
void launch_verify_blocks(const Batch& bt, cudaStream_t st);
// Copies n bytes with a kernel (no copy engine); one side may be mapped
// pinned host memory given by its device alias.  False (nothing launched)
// unless both addresses are 16-byte aligned.
bool launch_xfer(void* dst, const void* src, uint64_t n, cudaStream_t st);
void launch_block_decode(const Batch& bt, cudaStream_t st);
void launch_entries_from_offsets(const Batch& bt, cudaStream_t st);

// lc_merge.cu -- merge, drop rule, grandparent cuts, survivors
// the keys' common bytes, entry prefixes after them, grandparent prefixes
void launch_key_skip(const Batch& bt, cudaStream_t st);
void launch_merge(const Batch& bt, cudaStream_t st);
void launch_drop(const Batch& bt, cudaStream_t st);
void launch_triggers(const Batch& bt, cudaStream_t st);
void launch_kept_compact(const Batch& bt, cudaStream_t st);

// lc_encode.cu -- survivors -> output tables
void launch_sizes(const Batch& bt, cudaStream_t st);       // also clears the block starts
void launch_next(const Batch& bt, cudaStream_t st);
void launch_chain(const Batch& bt, cudaStream_t st);
void launch_block_list(const Batch& bt, cudaStream_t st);  // also the block sizes
void launch_files(const Batch& bt, cudaStream_t st);
void launch_block_layout(const Batch& bt, cudaStream_t st);
void launch_file_layout(const Batch& bt, cudaStream_t st);
// after the layout, blocks / filters / index + file keys are independent
void launch_encode_blocks(const Batch& bt, cudaStream_t st);
void launch_encode_filters(const Batch& bt, cudaStream_t st);
// the decoded form of the survivors, for jobs with keep_decoded
void launch_emit_decoded(const Batch& bt, cudaStream_t st);
void launch_encode_index(const Batch& bt, cudaStream_t st);
// metaindex, footer, filter tails and the trailers of filter/meta/index
void launch_encode_meta(const Batch& bt, cudaStream_t st);

// grid x for a kernel over up to `items` items per job, `per` items per CTA,
// capped at `cap` CTAs (the kernel loops over the rest)
inline unsigned grid_x(uint64_t items, unsigned per, uint64_t cap) {
  uint64_t g = (items + per - 1) / per;
  if (g == 0) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

}  // namespace lc
