/*
 * luda_b200 -- B200 (sm_100a) LSM compaction engine, C ABI.
 *
 * This is the boundary a LevelDB host calls in place of the body of
 * DBImpl::DoCompactionWork (reference: db/db_impl.cc:1060 for the CPU version
 * and db/db_impl.cc:1229 for LUDA's GPU version).  The version set, MANIFEST
 * edits, file numbering and file I/O stay in the host; the engine receives the
 * bytes of the input tables plus the few pieces of version state the
 * compaction loop reads, and returns the bytes of the output tables, which are
 * byte-identical to what the reference's CPU DoCompactionWork would write.
 *
 * All entry points are extern "C", take plain pointers and sizes, never throw,
 * and return an lc_status.  Nothing here is thread-safe unless stated.
 */
#ifndef LUDA_B200_H_
#define LUDA_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference returns leveldb::Status; LC_ERR_CORRUPT maps to
 * Status::Corruption, LC_ERR_INVALID_ARG to Status::InvalidArgument and the
 * rest to Status::IOError in the host shim. */
typedef enum {
  LC_OK = 0,
  LC_ERR_INVALID_ARG = 1, /* bad descriptor, option or handle */
  LC_ERR_CORRUPT = 2,     /* an input table failed a format check, or a merge
                           * child's entries are out of internal-key order */
  LC_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  LC_ERR_NO_MEMORY = 4,   /* device or host allocation failed */
  LC_ERR_BUDGET = 5,      /* job larger than the engine's device budget */
  LC_ERR_TIMEOUT = 6,     /* lc_job_wait timed out, or a device wait gave up */
  LC_ERR_UNSUPPORTED = 7, /* input beyond an engine limit (a job of 4 GiB or more,
                           * a key of 64 KiB or more) */
  LC_ERR_SHUTDOWN = 8     /* engine is being destroyed */
} lc_status;

typedef struct lc_engine lc_engine;
typedef struct lc_job lc_job;
/* The decoded entries of one output table, kept in device memory by the job
 * that wrote the table (lc_job_desc.keep_decoded) and valid until that job is
 * released.  Opaque. */
typedef struct lc_decoded lc_decoded;

typedef struct {
  int32_t device;               /* CUDA device ordinal */
  uint64_t device_budget_bytes; /* admission budget; 0 = 40 GiB */
  int32_t max_inflight_jobs;    /* worker threads, i.e. batches on the device at once; 0 = 4 */
  uint32_t flags;               /* LC_FLAG_* */
  int32_t max_batch_jobs;       /* jobs one batch (one set of launches) may hold; 0 = 64 */
  uint64_t max_batch_bytes;     /* input bytes a worker gathers into one batch (a larger
                                   job still runs, alone); 0 = 512 MiB */
  uint64_t pinned_reserve_bytes;/* pinned host memory for job outputs taken up front (more
                                   is added on demand in slabs of >= 256 MiB); 0 = none */
} lc_config;

/* lc_config.flags: record CUDA events around each phase of every job on the
 * job's own stream and report the device time per phase in lc_job_out. */
#define LC_FLAG_PHASE_TIMING 1u
/* lc_config.flags: launch every kernel directly instead of replaying captured
 * CUDA graphs (same results; for debugging and for measuring the graphs). */
#define LC_FLAG_NO_GRAPHS 2u

/* One input SSTable (the bytes of a file at level L or L+1). */
typedef struct {
  const uint8_t* data; /* host pointer, or device pointer if inputs_on_device */
  uint64_t size;       /* FileMetaData::file_size */
} lc_table;

/* A file at a level >= L+2, by key range (FileMetaData, db/version_edit.h:18). */
typedef struct {
  const uint8_t* smallest; /* internal key, host memory */
  uint32_t smallest_len;
  const uint8_t* largest; /* internal key, host memory */
  uint32_t largest_len;
  uint64_t file_size;
  int32_t level;
} lc_file_range;

/* The Options fields that shape output bytes (include/leveldb/options.h). */
typedef struct {
  uint32_t block_size;       /* Options::block_size */
  uint32_t restart_interval; /* Options::block_restart_interval */
  int32_t bits_per_key;      /* NewBloomFilterPolicy(bits_per_key); <= 0: no filter */
  uint64_t max_file_size;    /* Compaction::MaxOutputFileSize() */
} lc_table_options;

/* One compaction.  Replaces the CompactionState* argument of
 * DBImpl::DoCompactionWork (db/db_impl.cc:1060): the tables are those of
 * Compaction::inputs_[0] and inputs_[1] (db/version_set.h:380) in the order
 * VersionSet::MakeInputIterator makes merge children (db/version_set.cc:
 * 1237-1268): one child ("run") per level-0 file, one run per level >= 1
 * holding that level's files in key order. */
typedef struct {
  int32_t level;            /* Compaction::level() */
  int32_t n_tables;         /* all input tables, run-major */
  const lc_table* tables;
  int32_t n_runs;           /* merge children */
  const int32_t* run_table_count; /* tables per run, sums to n_tables */
  int32_t n_grandparents;   /* Compaction::grandparents_ (db/version_set.cc:1446) */
  const lc_file_range* grandparents;
  int32_t n_base_files;     /* every file at levels >= L+2, by level then key,
                               for Compaction::IsBaseLevelForKey (:1535) */
  const lc_file_range* base_files;
  uint64_t smallest_snapshot; /* CompactionState::smallest_snapshot (db/db_impl.cc:1073) */
  lc_table_options options;
  int32_t inputs_on_device; /* 1: lc_table.data are device pointers on the engine's device */
  int32_t outputs_on_device;/* 0: copy the output bytes to host memory;
                               1: leave them on the device only (lc_job_out.data is a
                               device pointer); 2: both -- host copy in data, device
                               copy in device_data, e.g. to feed a later job's
                               inputs_on_device without crossing PCIe again */
  int32_t verify_checksums; /* 1: check every input data block's CRC32C trailer on the
                               device before parsing it, and fail the job with
                               LC_ERR_CORRUPT ("block checksum mismatch") if one is
                               wrong -- ReadOptions::verify_checksums, which LevelDB
                               sets for compaction inputs from Options::paranoid_checks
                               (db/version_set.cc:1239; the check is table/format.cc:
                               86-95, switched off in the reference build).  0: no
                               check, as the reference. */
  int32_t keep_decoded;     /* 1 (with outputs_on_device 1 or 2): also keep every output
                               table's decoded entries in device memory
                               (lc_job_out.decoded), so that a later job reading that
                               table from device memory can skip parsing and decoding
                               it.  LUDA's nearest counterpart keeps a level-0 flush's
                               decoded entries in host memory for the compaction that
                               reads that file next (cuda/cuda_common.h:253-255, 339-355;
                               db/db_impl.cc:146-149). */
  const lc_decoded* const* decoded; /* NULL, or n_tables entries: for table i, the
                               decoded form of that same table (an lc_job_out.decoded
                               entry of the job that wrote it; NULL where none).  The
                               table must then be read from device memory
                               (inputs_on_device) and have the size the decoded form
                               was made for.  The output is byte-identical either way. */
} lc_job_desc;

/* Output of one compaction: what DoCompactionWork records in
 * CompactionState::outputs (db/db_impl.cc:197-201) plus the file bytes.  The
 * host assigns file numbers and writes the files.  All pointers stay valid
 * until lc_job_release. */
typedef struct {
  int32_t n_files;
  const uint8_t* data;          /* all output files back to back */
  const uint64_t* file_offset;  /* n_files, offset of file i in data */
  const uint64_t* file_size;    /* n_files */
  const uint64_t* file_entries; /* n_files, TableBuilder::NumEntries() */
  const uint8_t* key_bytes;     /* every file's smallest and largest internal keys (in
                                   fixed-size slots; use the offsets and lengths) */
  const uint64_t* smallest_offset; /* n_files: file i's smallest key is
                                      key_bytes[smallest_offset[i], + smallest_len[i]) */
  const uint32_t* smallest_len;
  const uint64_t* largest_offset;
  const uint32_t* largest_len;
  uint64_t bytes_in;    /* sum of input table sizes (CompactionStats::bytes_read) */
  uint64_t bytes_out;   /* sum of output sizes (CompactionStats::bytes_written) */
  uint64_t entries_in;  /* entries read */
  uint64_t entries_out; /* entries written */
  double device_ms;     /* device time of the job, first copy to last (CUDA events) */
  uint32_t kernel_launches; /* kernels the job launched */
  uint32_t n_phases;        /* > 0 with LC_FLAG_PHASE_TIMING */
  const char* const* phase_name;
  const float* phase_ms;    /* device time per phase */
  uint64_t key_bytes_in;    /* decoded internal-key bytes (input) */
  uint64_t value_bytes_out; /* value bytes written */
  uint64_t key_bytes_out;   /* internal-key bytes of the survivors */
  const uint8_t* device_data; /* outputs_on_device 1 or 2: the output bytes in device
                                 memory (same layout as data), else NULL */
  uint32_t batch_jobs;        /* jobs in the batch that ran this job (device_ms and
                                 kernel_launches are the batch's) */
  double queue_ms;            /* lc_job_submit -> start of its batch (0 for synchronous
                                 calls) */
  const lc_decoded* const* decoded; /* keep_decoded: n_files entries, the decoded entries
                                 of each output table (valid until lc_job_release);
                                 else NULL */
  uint32_t decoded_inputs;    /* input tables read from their decoded form */
} lc_job_out;

/* Engine lifetime.  An engine owns one CUDA device, its streams, slab caches
 * of device memory (batch scratch, outputs kept on the device) and of pinned
 * host memory (output copies), and a set of worker threads.  Release every
 * job handle before destroying the engine: the outputs live in its slabs. */
lc_status lc_engine_create(const lc_config* cfg, lc_engine** out);
void lc_engine_destroy(lc_engine* e);

/* Asynchronous jobs (thread-safe).  lc_job_submit copies the descriptor (not
 * the table bytes: host table buffers must stay valid until lc_job_wait
 * returns) and admits the job against the device budget; jobs beyond the
 * in-flight limit queue on the host.  lc_job_wait blocks until the job is done
 * or timeout_ns passes (< 0: forever). */
lc_status lc_job_submit(lc_engine* e, const lc_job_desc* desc, lc_job** out);
lc_status lc_job_wait(lc_job* j, int64_t timeout_ns);
lc_status lc_job_result(lc_job* j, lc_job_out* out);
/* Blocks until any of the n jobs (all of engine e) is done, or timeout_ns
 * passes (< 0: forever; LC_ERR_TIMEOUT), and stores its position in *index.
 * No counterpart in the reference (its compactions run one at a time on the
 * Env background thread): it is the completion queue of a request loop that
 * keeps many jobs in flight.  The finished job's own status comes from
 * lc_job_wait / lc_job_result. */
lc_status lc_job_wait_any(lc_engine* e, lc_job* const* jobs, int32_t n, int64_t timeout_ns,
                          int32_t* index);
/* Frees the job and its output buffers.  Device outputs (outputs_on_device 1
 * or 2) go back to the engine and may be handed to the next job at once, so
 * call it only after every kernel or copy of the caller's own that reads
 * them has completed. */
void lc_job_release(lc_job* j);

/* The device memory lc_job_submit admits a job with, against
 * lc_config.device_budget_bytes: the input copy (host inputs), the parse
 * arrays, the key arena, the output and the per-entry arrays, with the entry
 * count taken as one per 40 input bytes (it is known only after the parse;
 * a running batch then holds what it really allocated).  A job whose
 * estimate exceeds the budget is refused with LC_ERR_BUDGET.  No counterpart
 * in the reference, whose compactions run one at a time. */
lc_status lc_estimate_device_bytes(const lc_job_desc* desc, uint64_t* bytes);

/* Synchronous compaction on the calling thread: the drop-in for one
 * DoCompactionWork call.  *job_out must be released with lc_job_release. */
lc_status lc_compact(lc_engine* e, const lc_job_desc* desc, lc_job_out* out, lc_job** job_out);

/* Batched compaction (no counterpart in the reference, which runs one
 * DoCompactionWork at a time).  Runs n independent compactions together:
 * every kernel launch covers all jobs of a batch (up to max_batch_jobs; more
 * are split into several batches), and the kernel sequence after the first
 * host synchronisation is one captured CUDA graph, replayed for later batches
 * of the same shape.  When more than 128 MiB of the inputs are in host
 * memory, the jobs run as about eight batches (in order) on four streams at
 * once, so that host<->device copies overlap kernels; the call returns when
 * all have finished.  Each job's output is byte-identical to lc_compact on the
 * same descriptor.  On return every jobs[i] is a finished handle (release each
 * with lc_job_release): lc_job_wait returns its status at once and
 * lc_job_result its output.  Returns LC_OK when every job succeeded, else the
 * status of the first job that failed; argument errors create no handles. */
lc_status lc_compact_batch(lc_engine* e, int32_t n, const lc_job_desc* descs, lc_job** jobs);

/* Engine counters (no counterpart in the reference; the nearest is the
 * per-level CompactionStats behind GetProperty("leveldb.stats"),
 * db/db_impl.cc:1930). */
typedef struct {
  uint64_t batches;          /* batches run (a synchronous compaction is one) */
  uint64_t jobs;             /* compaction jobs run */
  uint64_t graph_captures;   /* kernel sequences captured into a new CUDA graph */
  uint64_t graph_replays;    /* batches that replayed a cached graph */
  uint64_t direct_tails;     /* batches whose shape was new: kernels launched directly */
  uint64_t pinned_bytes;     /* pinned host memory held for outputs */
  uint64_t pinned_free_bytes;/* ... of which not in use */
  uint64_t inflight_bytes;   /* device-memory estimate of the admitted jobs */
  uint64_t queued_jobs;      /* submitted jobs not yet admitted */
  /* host-side costs, for finding stalls */
  uint64_t block_takes;      /* scratch chunks and kept outputs taken from the device slabs */
  uint64_t block_take_us;    /* host time in those takes (slab growth included) */
  uint64_t staging_grows;    /* per-slot pinned staging buffers re-allocated */
  uint64_t pinned_slab_grows;/* pinned output slabs added after creation */
  uint64_t setup_us_max;     /* longest host set-up of a batch before its first kernel */
  uint64_t exact_reruns;     /* jobs rerun with exact counting (single pass overflowed) */
  /* device memory: slabs taken from the driver, their free part, the most
   * of them in use at once, slabs added */
  uint64_t scratch_bytes, scratch_free_bytes, scratch_peak_bytes, scratch_slab_grows;
  uint64_t device_out_bytes, device_out_free_bytes, device_out_peak_bytes, device_out_slab_grows;
} lc_engine_stats;
lc_status lc_engine_get_stats(lc_engine* e, lc_engine_stats* out);

/* Launch parameters the autotuner chooses (no counterpart in the reference). */
typedef struct {
  uint32_t ctas_per_job;  /* CTAs per job in the grid-stride kernels; 0 = from the sizes */
  uint32_t merge_items;   /* merge-path outputs per thread, 1..32 */
  uint32_t merge_threads; /* threads per merge CTA: 64..1024, a multiple of 32;
                             the merge tile is merge_threads * merge_items outputs */
} lc_tuning;

lc_status lc_get_tuning(lc_engine* e, lc_tuning* out);
/* Applies to batches that start after the call. */
lc_status lc_set_tuning(lc_engine* e, const lc_tuning* t);

/* Autotuner: runs the n jobs as batches under candidate settings (merge
 * tile, items per thread, CTAs per job), `repeats` times each, keeps the one
 * with the lowest median device time for the engine and writes it to
 * *chosen.  The outputs are computed and discarded; the descriptors' inputs
 * must stay valid for the call. */
lc_status lc_autotune(lc_engine* e, int32_t n, const lc_job_desc* descs, int32_t repeats,
                      lc_tuning* chosen);

/* Flush encoder: one table from n sorted internal keys and values, the GPU
 * counterpart of BuildTable's TableBuilder loop (db/builder.cc:17-60; LUDA's
 * GPUWriteLevel0, db/db_impl.cc:86-181).  Keys/values are packed with n+1
 * offsets, all in host memory (or device memory if on_device).  The table is
 * returned like a one-file compaction output (no size split). */
lc_status lc_build_table(lc_engine* e, const lc_table_options* opt, int64_t n,
                         const uint8_t* keys, const uint64_t* key_offsets,
                         const uint8_t* values, const uint64_t* value_offsets,
                         int32_t on_device, lc_job_out* out, lc_job** job_out);

/* Masked CRC32C of one buffer: crc32c::Mask(crc32c::Value(data, n))
 * (util/crc32c.h:20-32), the value LevelDB stores in a block trailer
 * (table/table_builder.cc:186-189) and that ReadBlock's verify_checksums path
 * checks (table/format.cc:87-94).  Computed on the engine's device over many
 * CTAs; data is host memory (copied in) or, with on_device, device memory.
 * The result is written to *masked_crc (host memory).  Scratch comes from the
 * engine's device memory pool. */
lc_status lc_crc32c(lc_engine* e, const uint8_t* data, uint64_t n, int32_t on_device,
                    uint32_t* masked_crc);

/* Allocation-free masked CRC32C.  No counterpart in the reference: it exists
 * for hosts that cannot allocate device memory at the moment they need a
 * checksum -- for example a host whose device memory is entirely owned by
 * another allocator, or a path that must not take the device-wide
 * synchronisation cudaMalloc/cudaFree imply.  It computes the same value as
 * lc_crc32c, needs no engine, takes device pointers only (d_data: n input
 * bytes; d_masked_crc: 4 output bytes), runs on `stream` (a cudaStream_t, or
 * NULL for the default stream) and returns without waiting for the GPU.
 *
 * Scratch is one fixed static device array (about 64 KiB, held by every
 * device that loads the library until the process exits), so n is limited to
 * 1 GiB; larger buffers are rejected with LC_ERR_UNSUPPORTED before anything
 * is launched.  Null pointers give LC_ERR_INVALID_ARG, runtime failures
 * LC_ERR_CUDA; each failure also sets lc_last_error().  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current and keeps it; make that first call before any stream capture,
 * and do not use the entry point across a cudaDeviceReset (the kept address
 * belongs to the context that was reset).  Every call clears the part of the array that must
 * start at zero, but all calls share the array: calls that overlap on the GPU
 * (on different streams, or from different threads) race, so serialise them,
 * e.g. on one stream. */
lc_status lc_crc32c_noalloc(const uint8_t* d_data, uint64_t n, uint32_t* d_masked_crc,
                            void* stream);

/* Human-readable message for the last error on this engine (thread-local). */
const char* lc_last_error(void);
const char* lc_status_string(lc_status s);

/* Library version. */
const char* lc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LUDA_B200_H_ */
