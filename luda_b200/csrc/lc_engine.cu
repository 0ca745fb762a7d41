// Host orchestration and the C ABI (include/luda_b200.h).
//
// Jobs run in batches; a plain compaction is a batch of one.  Every kernel
// launch covers all jobs of the batch (grid y = job), so a batch costs the
// same number of launches and host synchronisations as one job:
//   upload -> table/index parse -> [checksums] -> entry counts
//   -> [sync: entry totals]
//   -> decode -> merge rounds -> drop rule + grandparent cuts -> survivors
//   -> entry sizes -> block chain -> blocks -> files -> layout -> encode
//      (one captured CUDA graph, replayed for later batches of the same shape)
//   -> [sync: file counts and output sizes] -> download -> [sync]
// Device memory for a batch's working arrays and for outputs kept on the
// device comes from engine-wide slab caches (SlabCache), reused at once
// across the workers' streams; the CRC entry points use the stream-ordered
// pool, whose release threshold is raised so freed blocks are reused.
// Asynchronous jobs are served by worker threads, each with its own stream,
// descriptor array and graph cache; a worker takes every queued job that fits
// the device budget as one batch, so jobs that arrive while a batch runs are
// admitted into the next one (continuous batching).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/luda_b200.h"
#include "lc_crc_chunks.cuh"
#include "lc_device.cuh"
#include "lc_job.h"
#include "lc_kernels.h"

using namespace lc;

namespace {

thread_local std::string g_last_error;

const char* kVersion = "luda_b200 0.1 (sm_100a)";
constexpr uint32_t kCrcXpowN = 8192;
constexpr uint32_t kChunk = 4096;

struct CudaError {
  cudaError_t e;
  const char* what;
};

#define CK(call)                                   \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) throw CudaError{_e, #call}; \
  } while (0)

struct StatusError {
  lc_status s;
  std::string msg;
};

uint64_t round16(uint64_t x) { return (x + 15) & ~uint64_t(15); }

// A host<->device copy as pieces of `piece` bytes.  Jobs' host copies run one
// job at a time per direction (CopyLane), so an upload shares the link only
// with one download.  Measured on B200 with an upload and a download of 1 GiB
// each in flight at once: pieces of 2 MiB moved 40 + 40 GB/s, of 16 MiB
// 46 + 49, whole copies 50 + 51 (55 and 57 GB/s each alone).  A copy engine
// takes one piece at a time, so the next job's copies in the same direction
// wait up to one piece: piece_for() keeps a piece at about a sixteenth of
// the job's bytes (64 MiB pieces had slowed pipelined 66 MiB jobs by half).
void copy_pieces(void* dst, const void* src, uint64_t n, cudaMemcpyKind kind, cudaStream_t st,
                 uint64_t piece) {
  if (kind == cudaMemcpyDeviceToDevice) {
    CK(cudaMemcpyAsync(dst, src, n, kind, st));
    return;
  }
  for (uint64_t o = 0; o < n; o += piece)
    CK(cudaMemcpyAsync((uint8_t*)dst + o, (const uint8_t*)src + o, std::min(piece, n - o), kind, st));
}
uint64_t piece_for(uint64_t job_bytes) {
  uint64_t p = 2ull << 20;
  while (p < (64ull << 20) && p * 2 <= job_bytes / 16) p *= 2;
  return p;
}

// Memory for job outputs and scratch, pinned host memory or device memory.  Taking
// memory from the driver costs milliseconds (page locking; device mappings,
// which also hold up the other threads' CUDA calls), far more than a small
// job's device time, so it is taken in slabs of at least 256 MiB and handed
// out by first fit from a free list with neighbour coalescing; it returns to
// the driver only when the engine is destroyed.  A returned block is free for
// the next job at once, on any stream: the engine returns scratch and outputs
// only after the batch that used them has completed, and a caller returns an
// output (lc_job_release) only after its own reads of it have completed.
// (Scratch used to come from the stream-ordered pool: a batch bigger than any
// before made the pool map fresh memory in the middle of the batch, ~0.4 s
// for a few GB, holding up every other thread's CUDA calls meanwhile.)
struct SlabCache {
  static constexpr uint64_t kAlign = 4096;
  const bool device;      // device memory (cudaMalloc) rather than pinned host memory
  const uint64_t kSlab;   // smallest slab taken from the driver
  SlabCache(bool dev, uint64_t min_slab) : device(dev), kSlab(min_slab) {}
  std::mutex mu;
  std::vector<std::pair<uint8_t*, uint64_t>> slabs;
  std::map<uint8_t*, uint64_t> free_blocks;  // start -> size, address order
  uint64_t total = 0;                         // bytes in slabs
  std::atomic<uint64_t> grows{0};             // slabs added by take()
  uint64_t in_use = 0, peak = 0;              // bytes handed out: now, at most
  uint8_t* take(uint64_t n, uint64_t* cap) {
    const uint64_t want = (std::max<uint64_t>(n, 1) + kAlign - 1) & ~(kAlign - 1);
    while (true) {
      uint64_t grow;
      {
        std::lock_guard<std::mutex> g(mu);
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
          if (it->second < want) continue;
          uint8_t* p = it->first;
          const uint64_t rest = it->second - want;
          free_blocks.erase(it);
          if (rest) free_blocks.emplace(p + want, rest);
          *cap = want;
          in_use += want;
          peak = std::max(peak, in_use);
          return p;
        }
        // host: grow geometrically, so that a growing working set pins few
        // slabs; device: by a slab at a time, device memory being scarcer
        grow = std::max(kSlab, want);
        if (!device) grow = std::max(grow, total / 2);
      }
      // taking memory from the driver takes milliseconds: not under the
      // lock, so that returns (give) and other takes proceed meanwhile
      if (!add_slab(grow)) return nullptr;
      grows++;
    }
  }
  bool add_slab(uint64_t sz) {
    void* p = nullptr;
    if ((device ? cudaMalloc(&p, sz) : cudaMallocHost(&p, sz)) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    std::lock_guard<std::mutex> g(mu);
    slabs.emplace_back((uint8_t*)p, sz);
    free_blocks.emplace((uint8_t*)p, sz);
    total += sz;
    return true;
  }
  void give(uint8_t* p, uint64_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> g(mu);
    in_use -= cap;
    auto it = free_blocks.emplace(p, cap).first;
    // merge with the following block, then with the preceding one, when they
    // touch within one slab (two slabs may be adjacent in the address space,
    // but each goes back to the driver on its own)
    auto nx = std::next(it);
    if (nx != free_blocks.end() && it->first + it->second == nx->first &&
        same_slab(it->first, nx->first)) {
      it->second += nx->second;
      free_blocks.erase(nx);
    }
    if (it != free_blocks.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first && same_slab(pv->first, it->first)) {
        pv->second += it->second;
        free_blocks.erase(it);
      }
    }
  }
  bool same_slab(const uint8_t* a, const uint8_t* b) const {
    for (auto& sl : slabs)
      if (a >= sl.first && a < sl.first + sl.second) return b >= sl.first && b < sl.first + sl.second;
    return false;
  }
  void clear() {
    std::lock_guard<std::mutex> g(mu);
    for (auto& sl : slabs) device ? cudaFree(sl.first) : cudaFreeHost(sl.first);
    slabs.clear();
    free_blocks.clear();
    total = 0;
  }
};

struct Tunables {
  uint32_t ctas_per_job = 0;     // grid x of the grid-stride kernels (0: from the sizes)
  uint32_t merge_items = 8;      // merge-path outputs per thread
  uint32_t merge_threads = 256;  // threads per merge CTA
};

}  // namespace

struct lc_slot;

struct lc_engine {
  int device = 0;
  uint64_t budget = 40ull << 30;
  int max_inflight = 4;
  uint32_t flags = 0;
  uint32_t* crc_xpow = nullptr;
  SlabCache pinned{false, 256ull << 20};  // outputs' host copies
  SlabCache dev_out{true, 256ull << 20};  // outputs kept on the device
  SlabCache scratch{true, 1ull << 30};    // the batches' working arrays
  std::mutex mu;
  std::condition_variable cv;
  std::condition_variable admit_cv;
  std::mutex done_mu;  // completion of any job (lc_job_wait_any)
  std::condition_variable done_cv;
  std::deque<lc_job*> queue;
  std::vector<std::thread> workers;
  bool stop = false;
  uint64_t inflight_bytes = 0;
  uint32_t max_batch = 64;
  uint64_t max_batch_bytes = 512ull << 20;
  bool use_graphs = true;
  std::mutex tun_mu;
  Tunables tun;
  // Host<->device copies of jobs from host buffers run one job at a time per
  // direction, in the order they are issued: each batch's uploads wait on an
  // event after the previous batch's uploads (downloads likewise), so that one
  // job's download overlaps the next one's upload at each direction's full
  // rate instead of several jobs sharing a direction and then idling it
  // together.
  struct CopyLane {
    std::mutex mu;
    cudaEvent_t done = nullptr;
    bool any = false;
  };
  CopyLane up_lane, down_lane;
  // one slot per worker thread, then slots for synchronous calls (grown on
  // demand, one per concurrent caller)
  std::vector<std::unique_ptr<lc_slot>> slots;
  std::mutex slot_mu;
  std::vector<lc_slot*> free_slots;
  // counters for lc_engine_get_stats
  std::atomic<uint64_t> n_batches{0}, n_jobs{0}, n_captures{0}, n_replays{0}, n_direct{0};
  std::atomic<uint64_t> n_block_takes{0}, block_take_ns{0}, n_staging_grows{0}, setup_ns_max{0};
  std::atomic<uint64_t> n_exact_reruns{0};
  void note_setup(std::chrono::steady_clock::time_point t0) {
    const uint64_t ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                            std::chrono::steady_clock::now() - t0).count();
    uint64_t cur = setup_ns_max.load();
    while (ns > cur && !setup_ns_max.compare_exchange_weak(cur, ns)) {
    }
  }
  // Adds delta to the device bytes admitted jobs hold (a batch trues up its
  // admission estimate once its entry counts are known); a decrease may
  // admit queued jobs.
  void adjust_inflight(int64_t delta) {
    if (!delta) return;
    {
      std::lock_guard<std::mutex> g(mu);
      inflight_bytes = (uint64_t)((int64_t)inflight_bytes + delta);
    }
    if (delta < 0) admit_cv.notify_all();
  }
  lc_slot* take_slot();
  void put_slot(lc_slot* s);
  Tunables tuning() {
    std::lock_guard<std::mutex> g(tun_mu);
    return tun;
  }
  ~lc_engine();
};

// A table's decoded entries, kept in device memory by the job that wrote the
// table (a view into that job's decoded buffer); released with that job.
struct lc_decoded {
  DecRun run;
  uint64_t table_size;
};

struct lc_job {
  lc_engine* eng = nullptr;
  int kind = 0;  // 0 compaction, 1 build table
  // descriptor copy
  int32_t level = 0;
  std::vector<lc_table> tables;
  std::vector<int32_t> run_counts;
  std::vector<std::string> gp_largest;
  std::vector<uint64_t> gp_size;
  std::vector<int32_t> base_level;
  std::vector<std::string> base_small, base_large;  // user keys
  uint64_t smallest_snapshot = 0;
  lc_table_options opt{};
  int32_t inputs_on_device = 0, outputs_on_device = 0;
  int32_t verify_checksums = 0;
  int32_t keep_decoded = 0;
  std::vector<const lc_decoded*> in_dec;  // per input table, or empty (none)
  uint8_t* d_dec = nullptr;               // the survivors' decoded form (keep_decoded)
  uint64_t d_dec_cap = 0;
  std::vector<lc_decoded> out_dec;        // per output file: views into d_dec
  std::vector<const lc_decoded*> out_dec_ptrs;
  uint32_t decoded_inputs = 0;
  // build-table inputs
  int64_t bn = 0;
  const uint8_t *bkeys = nullptr, *bvals = nullptr;
  const uint64_t *bkoffs = nullptr, *bvoffs = nullptr;
  // results
  lc_status status = LC_OK;
  std::string err;
  uint8_t* h_out = nullptr;
  uint64_t h_out_cap = 0;
  uint8_t* d_out = nullptr;  // kept when outputs_on_device is 1 or 2
  uint64_t d_out_cap = 0;    // its block in the engine's device slabs
  std::vector<uint64_t> file_offset, file_size, file_entries, small_off, large_off;
  std::vector<uint32_t> small_len, large_len;
  std::vector<uint8_t> key_bytes;
  uint64_t bytes_in = 0, bytes_out = 0, entries_in = 0, entries_out = 0;
  double device_ms = 0;
  uint32_t launches = 0;
  uint32_t batch_jobs = 1;
  std::chrono::steady_clock::time_point t_submit;
  double queue_ms = 0;  // submit -> start of the batch that ran it
  std::vector<float> phase_ms;
  uint64_t key_bytes_in = 0, kept_key_bytes = 0, kept_value_bytes = 0;
  uint64_t est_bytes = 0;
  // completion
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
};

namespace {

// Device allocations of one batch: a bump allocator over chunks of the
// engine's scratch slabs (64 MiB or one array, whichever is larger), all
// returned when the batch has completed.  Sub-allocations are 256-byte
// aligned and padded so that 16-byte vector loads may run past the end of an
// array.  Outputs that outlive the batch (kept on the device) come from the
// output slabs instead: their lifetimes are the caller's.
struct DevAlloc {
  static constexpr uint64_t kChunkBytes = 64ull << 20;
  cudaStream_t st;
  lc_engine* eng;
  std::vector<std::pair<uint8_t*, uint64_t>> chunks;  // from eng->scratch
  std::vector<std::pair<uint8_t*, uint64_t>> outs;    // from eng->dev_out
  uint8_t* cur = nullptr;
  uint64_t left = 0;
  uint64_t n_takes = 0, take_ns = 0;  // blocks taken and the host time it took
  uint64_t used = 0;                  // bytes of scratch chunks and outputs taken
  DevAlloc(cudaStream_t s, lc_engine* e) : st(s), eng(e) {}
  ~DevAlloc() {
    release({});
    eng->n_block_takes += n_takes;
    eng->block_take_ns += take_ns;
  }
  uint8_t* take(SlabCache& c, uint64_t n, uint64_t* cap, const char* what) {
    const auto t0 = std::chrono::steady_clock::now();
    uint8_t* p = c.take(n, cap);
    if (!p) {
      // the device's stream-ordered pool may hold the memory unused (it
      // keeps freed memory up to its release threshold): give that back and
      // retry once
      cudaDeviceSynchronize();
      cudaMemPool_t def = nullptr;
      if (cudaDeviceGetDefaultMemPool(&def, eng->device) == cudaSuccess) cudaMemPoolTrimTo(def, 0);
      p = c.take(n, cap);
      if (!p) throw CudaError{cudaErrorMemoryAllocation, what};
    }
    take_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                   std::chrono::steady_clock::now() - t0).count();
    n_takes++;
    return p;
  }
  template <typename T>
  T* get(uint64_t n) {
    const uint64_t bytes = (std::max<uint64_t>(n, 1) * sizeof(T) + 16 + 255) & ~uint64_t(255);
    if (bytes > left) {
      uint64_t cap = 0;
      cur = take(eng->scratch, std::max(bytes, kChunkBytes), &cap, "cudaMalloc (scratch slab)");
      chunks.emplace_back(cur, cap);
      left = cap;
      used += cap;
    }
    T* r = (T*)cur;
    cur += bytes;
    left -= bytes;
    return r;
  }
  // a job's output: from the output slabs when it outlives the batch
  uint8_t* output(uint64_t bytes, bool outlives) {
    if (!outlives) return get<uint8_t>(bytes + 64);
    uint64_t cap = 0;
    uint8_t* p = take(eng->dev_out, std::max<uint64_t>(bytes, 16) + 64, &cap,
                      "cudaMalloc (device output slab)");
    outs.emplace_back(p, cap);
    used += cap;
    return p;
  }
  // once the batch has completed: returns the part of output p past its
  // first `used` bytes to the slabs and gives the capacity it keeps
  uint64_t trim(const void* p, uint64_t used) {
    for (auto& o : outs) {
      if (o.first != p) continue;
      const uint64_t keep = (used + 64 + SlabCache::kAlign - 1) & ~(SlabCache::kAlign - 1);
      if (keep < o.second) {
        eng->dev_out.give(o.first + keep, o.second - keep);
        o.second = keep;
      }
      return o.second;
    }
    return 0;
  }
  // returns the scratch and the outputs not in `keep`, after the stream's
  // work (already complete on the normal path; an error path may still have
  // kernels in flight)
  void release(const std::vector<void*>& keep) {
    if (chunks.empty() && outs.empty()) return;
    cudaStreamSynchronize(st);
    for (auto& c : chunks) eng->scratch.give(c.first, c.second);
    chunks.clear();
    for (auto& o : outs)
      if (std::find(keep.begin(), keep.end(), (void*)o.first) == keep.end())
        eng->dev_out.give(o.first, o.second);
    outs.clear();
    cur = nullptr;
    left = 0;
  }
};


// Phases of a job, timed with CUDA events on the job's stream when the engine
// was created with LC_FLAG_PHASE_TIMING.
enum Phase : int {
  kUpload = 0, kParse, kDecode, kMerge, kDrop, kPartition, kEncodeBlocks, kEncodeMeta,
  kDownload, kNumPhases
};
const char* const kPhaseNames[kNumPhases] = {"upload", "parse", "decode", "merge", "drop",
                                             "partition", "encode_blocks", "encode_meta",
                                             "download"};

struct PhaseTimer {
  bool on = false;
  bool external = false;  // record as graph nodes while capturing
  cudaStream_t st = nullptr;
  std::vector<std::pair<int, cudaEvent_t>> evs;  // (phase ended here, or -1), in order
  std::vector<bool> owned;
  PhaseTimer(bool enable, cudaStream_t s) : on(enable), st(s) {}
  ~PhaseTimer() {
    for (size_t i = 0; i < evs.size(); i++)
      if (owned[i]) cudaEventDestroy(evs[i].second);
  }
  void record(int tag) {
    if (!on) return;
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    if (external) CK(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
    else CK(cudaEventRecord(e, st));
    evs.emplace_back(tag, e);
    owned.push_back(true);
  }
  // a phase runs from the previous recorded event to its mark
  void start() { record(-1); }
  void mark(int p) { record(p); }
  // events recorded by a replayed graph (owned by the graph)
  void borrow(const std::vector<std::pair<int, cudaEvent_t>>& g) {
    for (auto& e : g) {
      evs.push_back(e);
      owned.push_back(false);
    }
  }
  // hands the recorded events over (to a graph cache entry)
  std::vector<std::pair<int, cudaEvent_t>> take() {
    auto r = evs;
    evs.clear();
    owned.clear();
    return r;
  }
  void collect(std::vector<float>& out) {
    out.assign(kNumPhases, 0.f);
    if (!on) return;
    for (size_t i = 1; i < evs.size(); i++) {
      if (evs[i].first < 0) continue;
      float ms = 0;
      cudaEventElapsedTime(&ms, evs[i - 1].second, evs[i].second);
      out[evs[i].first] += ms;
    }
  }
};

const char* err_name(uint32_t code) {
  switch (code) {
    case kErrBadFooter: return "bad table footer";
    case kErrBadIndex: return "bad index block";
    case kErrBadBlock: return "bad data block";
    case kErrBadEntry: return "bad entry";
    case kErrShortKey: return "internal key shorter than 8 bytes";
    case kErrArenaOverflow: return "key arena overflow";
    case kErrRetryExact: return "single-pass key arena too small";
    case kErrLimit: return "engine limit exceeded";
    case kErrChecksum: return "block checksum mismatch";
    case kErrUnsorted: return "input entries out of internal-key order";
    default: return "unknown";
  }
}

uint32_t bloom_k(int bpk) {
  // util/bloom.cc:20-24
  size_t k = static_cast<size_t>(bpk * 0.69);
  if (k < 1) k = 1;
  if (k > 30) k = 30;
  return (uint32_t)k;
}

// Survivors (k_koff..k_vlen, counters n_kept / n_triggers set) -> encoded files.
void fill_common(JobDev& J, const lc_job* j, lc_engine* e) {
  memset(&J, 0, sizeof(J));
  J.block_size = j->opt.block_size;
  J.restart_interval = j->opt.restart_interval;
  J.bits_per_key = j->opt.bits_per_key;
  J.bloom_k = j->opt.bits_per_key > 0 ? bloom_k(j->opt.bits_per_key) : 0;
  J.max_file_size = j->opt.max_file_size;
  J.smallest_snapshot = j->smallest_snapshot;
  J.verify_checksums = j->verify_checksums ? 1u : 0u;
  J.max_gp_overlap = (int64_t)(10 * j->opt.max_file_size);  // db/version_set.cc:31-33
  J.crc_xpow = e->crc_xpow;
  J.crc_xpow_n = kCrcXpowN;
  J.crc_h5 = e->crc_xpow + kCrcXpowN;
  J.crc_xinv = J.crc_h5 + kCrcH5Words;
  J.crc_byte = J.crc_xinv + kCrcXinvN;
  J.crc_ones = J.crc_byte + 256;
  J.crc_xpow_hi = J.crc_ones + kCrcXpowN;
  J.chunk = kChunk;
  J.chain_smem_words = 11 * 1024;  // 44 KiB (static shared memory takes the rest of 48)
}

uint32_t ceil_log2(uint64_t x) {
  uint32_t r = 0;
  while ((1ull << r) < x) r++;
  return r;
}
uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Host-side state of one job inside a batch.
struct JobRun {
  lc_job* j = nullptr;
  JobDev J;
  uint64_t cap_blk = 0, N = 0, K = 0;
  // the input's bytes (tables rounded to 16), which bound the capacities; a
  // job reading device tables in place may span more address range than this
  uint64_t in_bytes = 0;
  uint32_t max_klen = 8;
  bool failed = false;
  Counters hc{};
  std::vector<FileOut> files;
  std::vector<uint64_t> koff;
  uint8_t* dec_block = nullptr;  // keep_decoded: the decoded buffer (device output slab)
  uint64_t dec_cap = 0;
};

void job_fail(JobRun& r, lc_status s, const std::string& m) {
  if (r.failed) return;
  r.failed = true;
  r.j->status = s;
  r.j->err = m;
}

lc_status counters_status(const Counters& c, std::string* msg) {
  if (!c.error) return LC_OK;
  *msg = std::string(err_name(c.error)) + " (detail " + std::to_string(c.error_detail) + ")";
  return (c.error == kErrLimit || c.error == kErrArenaOverflow) ? LC_ERR_UNSUPPORTED : LC_ERR_CORRUPT;
}

// Small per-job host arrays packed into one staging buffer and uploaded with
// one copy; device pointers are fixed up after the upload address is known.
struct Stage {
  std::vector<uint8_t> h;
  template <typename T>
  uint64_t put(const T* p, uint64_t n) {
    const uint64_t off = (h.size() + 255) & ~uint64_t(255);
    h.resize(off + std::max<uint64_t>(n * sizeof(T), 1) + 16);
    if (n) memcpy(h.data() + off, p, n * sizeof(T));
    return off;
  }
};

// Kernel sequence after the first sync, shared by the compaction and the
// flush-encoder paths.  Capturable: launches only, no host-side waits.
void launch_tail(const Batch& bt, bool decode_merge, cudaStream_t st, PhaseTimer& T) {
  if (decode_merge) {
    launch_block_decode(bt, st);
    launch_key_skip(bt, st);
    T.mark(kDecode);
    launch_merge(bt, st);
    T.mark(kMerge);
    launch_drop(bt, st);
    launch_triggers(bt, st);
    scan_batch(kScanKeep, bt, bt.max_entries, st);
    launch_kept_compact(bt, st);
    T.mark(kDrop);
  }
  launch_sizes(bt, st);
  scan_batch(kScanKb, bt, bt.max_entries, st);
  launch_next(bt, st);
  launch_chain(bt, st);
  scan_batch(kScanBstart, bt, bt.max_entries, st);
  launch_block_list(bt, st);
  scan_batch(kScanBcum, bt, bt.max_entries, st);
  launch_files(bt, st);
  launch_block_layout(bt, st);
  scan_batch(kScanIcum, bt, bt.max_entries, st);
  scan_batch(kScanGcum, bt, bt.max_entries, st);
  launch_file_layout(bt, st);
  T.mark(kPartition);
  launch_encode_blocks(bt, st);
  launch_emit_decoded(bt, st);
  T.mark(kEncodeBlocks);
  launch_encode_filters(bt, st);
  launch_encode_index(bt, st);
  launch_encode_meta(bt, st);
  T.mark(kEncodeMeta);
}

// Allocates the post-parse arrays of one job from its entry count N (and key
// bytes K for the arena) and fills its descriptor.
void alloc_tail(JobRun& r, DevAlloc& A, bool with_merge) {
  JobDev& J = r.J;
  const uint64_t N = r.N;
  if (with_merge) {
    J.keys = A.get<uint8_t>(r.K + 16);
    J.cap_key_bytes = r.K;
    J.cap_entries = N;
    J.e_rec = A.get<uint4>(N);
    J.e_koff = A.get<uint32_t>(N + 1);  // + the total (the scan of the key lengths)
    J.e_klen = A.get<uint32_t>(N);
    J.e_voff = A.get<uint32_t>(N);
    J.e_vlen = A.get<uint32_t>(N);
    J.e_pfx = A.get<uint64_t>(N);
    J.e_tag = A.get<uint64_t>(N);
    J.m_ids = A.get<uint32_t>(N);
    J.m_tmp = A.get<uint32_t>(N);
    J.m_pfx = A.get<uint64_t>(N);
    J.m_pfx_tmp = A.get<uint64_t>(N);
    J.m_tag = A.get<uint64_t>(N);
    J.m_tag_tmp = A.get<uint64_t>(N);
    J.cap_merge_tiles = (uint32_t)merge_tile_capacity(N, J.n_runs);
    J.m_split = A.get<uint32_t>(J.cap_merge_tiles);
    J.keep = A.get<uint8_t>(N);
    J.gp_idx = A.get<uint32_t>(J.n_gp ? N : 1);
    J.kept_pos = A.get<uint32_t>(N + 1);
    J.gp_first = A.get<uint32_t>(J.n_gp + 1);
    J.gp_upfx = A.get<uint64_t>(J.n_gp + 1);
    J.gp_mode = A.get<uint8_t>(J.n_gp + 1);
    J.k_forced = A.get<uint8_t>(N + 1);
  }
  J.k_koff = A.get<uint32_t>(N);
  J.k_klen = A.get<uint32_t>(N);
  J.k_voff = A.get<uint32_t>(N);
  J.k_vlen = A.get<uint32_t>(N);
  J.cap_triggers = J.n_gp + 1;
  J.triggers = A.get<uint32_t>(J.cap_triggers);
  J.k_a = A.get<uint32_t>(N);
  J.k_b = A.get<uint32_t>(N);
  J.k_shared = A.get<uint32_t>(N);
  J.k_next = A.get<uint32_t>(N);
  J.k_bstart = A.get<uint8_t>(N + 1);
  J.k_block = A.get<uint32_t>(N + 1);
  const uint64_t chunks = (N + J.chunk - 1) / J.chunk + 1;
  J.chunk_table = A.get<uint32_t>(chunks * J.chunk);
  J.chunk_entry = A.get<uint32_t>(chunks);
  J.group_table = A.get<uint32_t>((chunks / kChainGroup + 1) * J.chunk);
  J.b_first = A.get<uint32_t>(N + 1);
  J.b_size = A.get<uint32_t>(N);
  J.tmp32 = A.get<uint32_t>(N);
  J.b_cum = A.get<uint64_t>(N + 1);
  J.cap_files = (uint32_t)std::min<uint64_t>(
      N + 1, 64 + J.cap_triggers +
                 (8 * (r.in_bytes + J.cap_key_bytes) + N * 64) / std::max<uint64_t>(1, J.max_file_size));
  J.files = A.get<FileOut>(J.cap_files);
  J.b_fnext = A.get<uint32_t>(N);
  J.t_blocks = A.get<uint32_t>(J.cap_triggers);
  J.t_kept = A.get<uint32_t>(J.cap_triggers);
  J.k_pb = A.get<uint64_t>(N + 1);
  J.b_file = A.get<uint32_t>(N);
  J.b_off = A.get<uint64_t>(N);
  J.b_isize = A.get<uint32_t>(N);
  J.b_icum = A.get<uint64_t>(N + 1);
  J.b_sep = A.get<uint32_t>(N);
  J.b_ilen = A.get<uint32_t>(N);
  J.b_gbytes = A.get<uint32_t>(N);
  J.b_gcum = A.get<uint64_t>(N + 1);
  J.b_gkeys = A.get<uint32_t>(N);
  // Output capacity, bounded without waiting for the layout: every survivor
  // costs at most its key, its value and 15 header bytes; every block at most
  // 4 bytes of restart word per entry, 9 bytes of count and trailer, one index
  // entry (its last key + 31; the blocks' last keys are distinct survivors, so
  // all of them together are at most the key bytes) and a filter share; every
  // file 256 bytes of metaindex, footer and trailers.  The layout kernel
  // checks the real size against it.
  const uint64_t bpk = J.bits_per_key > 0 ? (uint64_t)J.bits_per_key : 0;
  if (J.reserve_keys) {
    // single pass (key bytes unknown): the survivors re-encoded take about
    // the input's bytes; a job whose layout needs more is rerun with exact
    // counting and the bound below
    J.cap_out = r.in_bytes + r.in_bytes / 4 + N * (64 + (bpk + 7) / 8) +
                (uint64_t)J.cap_files * 256 + 65536;
  } else {
    J.cap_out = r.in_bytes + 3 * J.cap_key_bytes + N * (80 + (bpk + 7) / 8) +
                (uint64_t)J.cap_files * 256 + (r.in_bytes + J.cap_key_bytes) / 256 + 65536;
  }
  J.out = A.output(J.cap_out, r.j->outputs_on_device == 1 || r.j->outputs_on_device == 2);
  if (r.j->keep_decoded && !r.failed) {
    // the survivors' decoded form, kept with the outputs: keys (at most the
    // arena), key offsets, value lengths and places, prefixes, tags
    const uint64_t kcap = (J.cap_key_bytes + 16 + 255) & ~uint64_t(255);
    const uint64_t n8 = ((N + 1) * 8 + 255) & ~uint64_t(255), n4 = (N * 4 + 255) & ~uint64_t(255);
    const uint64_t bytes = kcap + 3 * n8 + 2 * n4;
    uint8_t* q = A.output(bytes, true);
    r.dec_block = q;
    r.dec_cap = A.outs.back().second;
    J.dec_keys = q;
    J.dec_kcum = reinterpret_cast<uint64_t*>(q + kcap);
    J.dec_pfx = reinterpret_cast<uint64_t*>(q + kcap + n8);
    J.dec_tag = reinterpret_cast<uint64_t*>(q + kcap + 2 * n8);
    J.dec_vlen = reinterpret_cast<uint32_t*>(q + kcap + 3 * n8);
    J.dec_vpos = reinterpret_cast<uint32_t*>(q + kcap + 3 * n8 + n4);
  }
  J.fkeys = A.get<uint8_t>(2ull * J.cap_files * r.max_klen + 1);
  J.fkey_stride = r.max_klen;
  J.fkoff = A.get<uint64_t>(2ull * J.cap_files + 1);
  J.cap_scan = N + 1;
  J.scan_scratch = A.get<uint64_t>(scan_scratch_elems(N + 1));
}

}  // namespace

// One set of device resources per thread that runs batches: a stream, a
// persistent device array of job descriptors (so that captured graphs can be
// replayed for other batches), and the graph cache.
struct lc_slot {
  cudaStream_t st = nullptr;
  JobDev* d_jobs = nullptr;
  uint32_t cap = 0;
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    uint64_t uses = 0;
    uint32_t launches = 0;  // kernels in the graph
    std::vector<std::pair<int, cudaEvent_t>> events;  // phase marks inside the graph
  };
  std::map<std::string, GraphEntry> graphs;
  uint64_t tick = 0;
  // Pinned host staging for the slot's small copies (descriptors, counters,
  // per-file results), so that they are asynchronous DMA; it grows only at
  // points where none of its copies is in flight, at least doubling.  An
  // outgrown buffer is kept until the slot is destroyed: cudaFreeHost waits
  // for the whole device, which would stall every other slot's batch.
  uint8_t* pin = nullptr;
  uint8_t* pin_dev = nullptr;  // its device alias (mapped pinned memory), or null
  size_t pin_cap = 0;
  std::vector<uint8_t*> pin_retired;
  std::atomic<uint64_t>* grow_count = nullptr;
  uint8_t* pinned(size_t n) {
    if (n > pin_cap) {
      const size_t c = std::max<size_t>(n, std::max<size_t>(4 << 20, 2 * pin_cap));
      uint8_t* q = nullptr;
      CK(cudaMallocHost(&q, c));
      if (pin) pin_retired.push_back(pin);
      pin = q;
      pin_cap = c;
      pin_dev = nullptr;
      if (cudaHostGetDevicePointer((void**)&pin_dev, q, 0) != cudaSuccess) {
        cudaGetLastError();
        pin_dev = nullptr;
      }
      if (grow_count) (*grow_count)++;
    }
    return pin;
  }
  // A small transfer between device memory and this staging buffer: a
  // kernel through the buffer's device alias when there is one (it does not
  // queue behind other streams' bulk copies), else cudaMemcpyAsync.
  void to_device(void* d, const uint8_t* h, size_t n) {
    if (!(pin_dev && launch_xfer(d, pin_dev + (h - pin), n, st)))
      CK(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, st));
  }
  void to_host(uint8_t* h, const void* d, size_t n) {
    if (!(pin_dev && launch_xfer(pin_dev + (h - pin), d, n, st)))
      CK(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, st));
  }
  void init(int device, uint32_t capacity) {
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cap = capacity;
    CK(cudaMalloc(&d_jobs, sizeof(JobDev) * cap));
  }
  void destroy() {
    for (auto& g : graphs) {
      cudaGraphExecDestroy(g.second.exec);
      for (auto& ev : g.second.events) cudaEventDestroy(ev.second);
    }
    graphs.clear();
    if (pin) cudaFreeHost(pin);
    for (uint8_t* q : pin_retired) cudaFreeHost(q);
    pin_retired.clear();
    pin = nullptr;
    pin_dev = nullptr;
    pin_cap = 0;
    if (d_jobs) cudaFree(d_jobs);
    if (st) cudaStreamDestroy(st);
    d_jobs = nullptr;
    st = nullptr;
  }
  std::map<std::string, uint32_t> seen;  // shape keys met without a graph
  // Launches the post-parse sequence for `bt`: replays the cached graph of
  // the same grid shapes, or captures one when the shape comes back a second
  // time (capturing and instantiating cost more than launching directly, so
  // a shape met once runs without a graph).  Returns 0 direct, 1 captured,
  // 2 replayed.
  int run_tail(const Batch& bt, bool decode_merge, bool use_graph, PhaseTimer& T) {
    if (!use_graph) {
      launch_tail(bt, decode_merge, st, T);
      CK(cudaGetLastError());
      return 0;
    }
    char key[256];
    snprintf(key, sizeof(key), "%d|%d|%u|%u|%u|%u|%u|%llu|%llu|%u|%u|%u|%u|%u|%u|%d", (int)T.on,
             (int)decode_merge, bt.B, bt.max_tables, bt.max_gp, bt.max_cap_triggers,
             bt.max_cap_files, (unsigned long long)bt.max_blocks_in,
             (unsigned long long)bt.max_entries, bt.merge_rounds, bt.chunk, bt.ctas_per_job,
             bt.merge_items, bt.merge_threads, bt.max_runs,
             (int)bt.any_keep_decoded);
    auto it = graphs.find(key);
    bool fresh = false;
    if (it == graphs.end()) {
      if (seen.size() > 1024) seen.clear();
      if (++seen[key] < 2) {
        launch_tail(bt, decode_merge, st, T);
        CK(cudaGetLastError());
        return 0;
      }
      seen.erase(key);
      if (graphs.size() >= 24) {  // evict the least recently used
        auto victim = graphs.begin();
        for (auto g = graphs.begin(); g != graphs.end(); ++g)
          if (g->second.uses < victim->second.uses) victim = g;
        cudaGraphExecDestroy(victim->second.exec);
        for (auto& ev : victim->second.events) cudaEventDestroy(ev.second);
        graphs.erase(victim);
      }
      cudaGraph_t g;
      PhaseTimer Tc(T.on, st);
      Tc.external = true;
      const uint32_t l0 = launches_on_this_thread();
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      launch_tail(bt, decode_merge, st, Tc);
      cudaError_t le = cudaGetLastError();
      cudaError_t ee = cudaStreamEndCapture(st, &g);
      CK(le);
      CK(ee);
      GraphEntry ge;
      ge.launches = launches_on_this_thread() - l0;  // counted once, at capture
      ge.events = Tc.take();
      cudaError_t ie = cudaGraphInstantiate(&ge.exec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        for (auto& ev : ge.events) cudaEventDestroy(ev.second);
        CK(ie);
      }
      it = graphs.emplace(key, ge).first;
      fresh = true;
    }
    it->second.uses = ++tick;
    CK(cudaGraphLaunch(it->second.exec, st));
    if (!fresh) note_launch(it->second.launches);
    T.borrow(it->second.events);
    return fresh ? 1 : 2;
  }
};

lc_slot* lc_engine::take_slot() {
  std::lock_guard<std::mutex> g(slot_mu);
  if (!free_slots.empty()) {
    lc_slot* r = free_slots.back();
    free_slots.pop_back();
    return r;
  }
  std::unique_ptr<lc_slot> n(new lc_slot());
  n->init(device, max_batch);
  n->grow_count = &n_staging_grows;
  slots.push_back(std::move(n));
  return slots.back().get();
}

void lc_engine::put_slot(lc_slot* s) {
  std::lock_guard<std::mutex> g(slot_mu);
  free_slots.push_back(s);
}

lc_engine::~lc_engine() {
  cudaSetDevice(device);
  for (auto& sl : slots) sl->destroy();
}

namespace {

// Runs a batch of compaction jobs (kind 0) on one slot.  Per-job failures are
// recorded in the job; CUDA failures fail the whole batch.
// Key arena of the single-pass decode: the input bytes (typical keys decode
// to well under the table bytes), and keys of at most kFastMaxKey bytes; a job
// beyond either is rerun with exact counting.
constexpr uint32_t kFastMaxKey = 256;

// Holds the difference between a batch's admitted estimate and the device
// memory it actually took in the engine's in-flight bytes until the batch
// has released its scratch.
struct InflightTrueUp {
  lc_engine* e;
  int64_t delta = 0;
  explicit InflightTrueUp(lc_engine* eng) : e(eng) {}
  void set(int64_t d) {
    e->adjust_inflight(d - delta);
    delta = d;
  }
  ~InflightTrueUp() { e->adjust_inflight(-delta); }
};

// `admitted`: the device bytes a worker charged for these jobs at admission
// (0 for synchronous calls, which are not admitted against the budget).
void run_batch(std::vector<lc_job*>& jobs, lc_slot& slot, const Tunables& tun,
               bool exact = false, uint64_t admitted = 0) {
  if (jobs.empty()) return;
  lc_engine* e = jobs[0]->eng;
  InflightTrueUp trueup(e);
  const auto t_setup0 = std::chrono::steady_clock::now();
  cudaStream_t st = slot.st;
  DevAlloc A(st, e);
  PhaseTimer T((e->flags & LC_FLAG_PHASE_TIMING) != 0, st);
  const uint32_t launches0 = launches_on_this_thread();
  const uint32_t B = (uint32_t)jobs.size();
  if (B > slot.cap) {  // callers split batches at the slot's capacity
    for (auto* j : jobs) {
      j->status = LC_ERR_INVALID_ARG;
      j->err = "batch larger than the engine's max_batch_jobs";
    }
    return;
  }
  std::vector<JobRun> runs(B);
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  try {
    CK(cudaEventRecord(ev0, st));
    T.start();
    // ---- set-up: descriptors, input placement, small arrays
    Stage S;
    uint64_t in_total = 0;
    std::vector<std::vector<TableDesc>> tds(B);
    std::vector<uint64_t> in_base(B, 0);
    std::vector<bool> zero_copy(B, false);
    struct Offs {
      uint64_t td, dec, gpk, gpo, gpp, lb, bk, bso, blo, bsl, bll;
    };
    std::vector<Offs> offs(B);
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      lc_job* j = jobs[i];
      r.j = j;
      fill_common(r.J, j, e);
      JobDev& J = r.J;
      const uint32_t nt = (uint32_t)j->tables.size();
      auto& td = tds[i];
      td.resize(nt);
      uint32_t run = 0, in_run = 0;
      for (uint32_t t = 0; t < nt; t++) {
        while (run < j->run_counts.size() && in_run >= (uint32_t)j->run_counts[run]) {
          run++;
          in_run = 0;
        }
        td[t].run = run;
        td[t].size = j->tables[t].size;
        td[t].cached = (!j->in_dec.empty() && j->in_dec[t]) ? 1u : 0u;
        in_run++;
      }
      J.n_tables = nt;
      J.n_runs = (uint32_t)j->run_counts.size();
      uint64_t in_size = 0;
      if (j->inputs_on_device) {
        uintptr_t lo = ~uintptr_t(0), hi = 0;
        for (auto& t : j->tables) {
          lo = std::min(lo, (uintptr_t)t.data);
          hi = std::max(hi, (uintptr_t)t.data + (uintptr_t)t.size);
        }
        if (nt && hi - lo < (1ull << 32)) {
          zero_copy[i] = true;
          J.in = (const uint8_t*)lo;
          in_size = hi - lo;
          for (uint32_t t = 0; t < nt; t++) td[t].off = (uintptr_t)j->tables[t].data - lo;
        }
      }
      if (!zero_copy[i]) {
        for (uint32_t t = 0; t < nt; t++) {
          td[t].off = in_size;
          in_size += round16(td[t].size);
        }
        if (in_size >= (1ull << 32)) {
          job_fail(r, LC_ERR_UNSUPPORTED, "input of one job must be below 4 GiB");
          in_size = 0;
        }
        in_base[i] = in_total;
        in_total += in_size + 16;
      }
      J.in_size = in_size;
      r.in_bytes = 0;
      if (!r.failed)
        for (auto& t : td) r.in_bytes += round16(t.size);
      uint64_t cap_blk = 1;
      for (auto& t : td) cap_blk += t.size / 13 + 1;
      r.cap_blk = cap_blk;
      // grandparents: largest keys, offsets, size prefix
      J.n_gp = (uint32_t)j->gp_largest.size();
      std::vector<uint64_t> gpo(J.n_gp + 1, 0), gpp(J.n_gp + 1, 0);
      std::string gpk;
      for (uint32_t g = 0; g < J.n_gp; g++) {
        const std::string& k = j->gp_largest[g];
        gpk += k;
        gpo[g + 1] = gpk.size();
        gpp[g + 1] = gpp[g] + j->gp_size[g];
      }
      // base-level files, grouped by level
      const uint32_t nb = (uint32_t)j->base_level.size();
      std::vector<uint32_t> lb;
      std::vector<uint64_t> so(nb), lo_(nb);
      std::vector<uint32_t> sl(nb), ll(nb);
      std::string bk;
      for (uint32_t f = 0; f < nb; f++) {
        if (f == 0 || j->base_level[f] != j->base_level[f - 1]) lb.push_back(f);
        so[f] = bk.size();
        sl[f] = (uint32_t)j->base_small[f].size();
        bk += j->base_small[f];
        lo_[f] = bk.size();
        ll[f] = (uint32_t)j->base_large[f].size();
        bk += j->base_large[f];
      }
      lb.push_back(nb);
      J.n_base_levels = nb ? (uint32_t)lb.size() - 1 : 0;
      Offs& o = offs[i];
      o.td = S.put(td.data(), nt);
      {
        std::vector<DecRun> dr(nt);
        memset(dr.data(), 0, sizeof(DecRun) * nt);
        for (uint32_t t = 0; t < nt; t++)
          if (td[t].cached) dr[t] = j->in_dec[t]->run;
        o.dec = S.put(dr.data(), nt);
      }
      o.gpk = S.put(gpk.data(), gpk.size());
      o.gpo = S.put(gpo.data(), gpo.size());
      o.gpp = S.put(gpp.data(), gpp.size());
      o.lb = S.put(lb.data(), lb.size());
      o.bk = S.put(bk.data(), bk.size());
      o.bso = S.put(so.data(), nb);
      o.blo = S.put(lo_.data(), nb);
      o.bsl = S.put(sl.data(), nb);
      o.bll = S.put(ll.data(), nb);
    }
    // pinned staging before the first sync: [stage | descriptors | counters]
    const size_t o_hj = (S.h.size() + 255) & ~size_t(255);
    const size_t o_hc = o_hj + ((sizeof(JobDev) * B + 255) & ~size_t(255));
    uint8_t* pin1 = slot.pinned(o_hc + sizeof(Counters) * B);
    memcpy(pin1, S.h.data(), S.h.size());
    uint8_t* d_stage = A.get<uint8_t>(S.h.size());
    slot.to_device(d_stage, pin1, S.h.size());  // not behind other jobs' bulk copies
    uint8_t* d_in_all = in_total ? A.get<uint8_t>(in_total) : nullptr;
    Counters* d_ctr = A.get<Counters>(B);
    CK(cudaMemsetAsync(d_ctr, 0, sizeof(Counters) * B, st));
    Batch bt;
    bt.d = slot.d_jobs;
    bt.B = B;
    bt.chunk = kChunk;
    bt.ctas_per_job = tun.ctas_per_job;
    bt.merge_items = tun.merge_items;
    bt.merge_threads = tun.merge_threads;
    bool host_up = false;
    for (uint32_t i = 0; i < B; i++)
      host_up = host_up || (!zero_copy[i] && !jobs[i]->inputs_on_device && !runs[i].failed);
    std::unique_lock<std::mutex> up_lk(e->up_lane.mu, std::defer_lock);
    if (host_up) {
      up_lk.lock();
      if (e->up_lane.any) CK(cudaStreamWaitEvent(st, e->up_lane.done, 0));
    }
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      JobDev& J = r.J;
      lc_job* j = jobs[i];
      const Offs& o = offs[i];
      if (!zero_copy[i]) {
        J.in = d_in_all + in_base[i];
        for (uint32_t t = 0; t < J.n_tables && !r.failed; t++) {
          if (!j->tables[t].size) continue;
          copy_pieces((uint8_t*)J.in + tds[i][t].off, j->tables[t].data, j->tables[t].size,
                      j->inputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st,
                      piece_for(J.in_size));
        }
      }
      J.in_end = J.in + J.in_size + (zero_copy[i] ? 0 : 16);
      J.tables = (const TableDesc*)(d_stage + o.td);
      J.dec_runs = (const DecRun*)(d_stage + o.dec);
      J.gp_keys = d_stage + o.gpk;
      J.gp_key_off = (const uint64_t*)(d_stage + o.gpo);
      J.gp_prefix = (const uint64_t*)(d_stage + o.gpp);
      J.base_level_begin = (const uint32_t*)(d_stage + o.lb);
      J.base_keys = d_stage + o.bk;
      J.base_small_off = (const uint64_t*)(d_stage + o.bso);
      J.base_large_off = (const uint64_t*)(d_stage + o.blo);
      J.base_small_len = (const uint32_t*)(d_stage + o.bsl);
      J.base_large_len = (const uint32_t*)(d_stage + o.bll);
      J.ctr = d_ctr + i;
      if (r.failed) {
        J.n_tables = 0;
        J.n_runs = 0;
      }
      const uint64_t cap_blk = r.cap_blk;
      J.cap_blocks_in = cap_blk;
      J.tbl_nblocks = A.get<uint32_t>(J.n_tables);
      J.tbl_unit = A.get<uint32_t>(J.n_tables);
      J.tbl_block_base = A.get<uint64_t>(J.n_tables + 1);
      J.blk_off = A.get<uint64_t>(cap_blk);
      J.blk_size = A.get<uint32_t>(cap_blk);
      J.blk_run = A.get<uint32_t>(cap_blk);
      J.blk_nent = A.get<uint32_t>(cap_blk);
      J.blk_ent_base = A.get<uint64_t>(cap_blk + 1);
      J.blk_kbytes = A.get<uint64_t>(cap_blk);
      J.blk_key_base = A.get<uint64_t>(cap_blk + 1);
      J.scan_scratch = A.get<uint64_t>(scan_scratch_elems(cap_blk + J.n_tables + 1));
      J.run_entry_begin_w = A.get<uint64_t>(J.n_runs + 1);
      J.run_entry_begin = J.run_entry_begin_w;
      bt.max_tables = std::max(bt.max_tables, J.n_tables);
      bt.any_verify = bt.any_verify || (J.verify_checksums && !r.failed);
      bt.any_keep_decoded = bt.any_keep_decoded || (j->keep_decoded && !r.failed);
      bt.max_blocks_in = std::max(bt.max_blocks_in, cap_blk);
    }
    if (host_up) {
      CK(cudaEventRecord(e->up_lane.done, st));
      e->up_lane.any = true;
      up_lk.unlock();
    }
    JobDev* hj = reinterpret_cast<JobDev*>(pin1 + o_hj);
    for (uint32_t i = 0; i < B; i++) hj[i] = runs[i].J;
    slot.to_device(slot.d_jobs, (const uint8_t*)hj, sizeof(JobDev) * B);
    T.mark(kUpload);
    e->note_setup(t_setup0);
    // ---- parse: index blocks, then entry counts -- exact: a walk of every
    // entry header, which also gives the key bytes; single pass: the restart
    // words alone, the decode reserving key space itself
    if (bt.max_tables) {
      launch_table_index_count(bt, st);
      scan_batch(kScanTblBlocks, bt, bt.max_tables, st);
      launch_table_index_entries(bt, st);
      launch_verify_blocks(bt, st);
      if (exact) {
        launch_block_count(bt, st);
        scan_batch(kScanBlkEnt, bt, bt.max_blocks_in, st);
        scan_batch(kScanBlkKey, bt, bt.max_blocks_in, st);
      } else {
        launch_block_restarts(bt, st);
        scan_batch(kScanBlkEnt, bt, bt.max_blocks_in, st);
      }
    }
    launch_run_bounds(bt, st);
    CK(cudaGetLastError());
    T.mark(kParse);
    std::vector<Counters> hc(B);
    slot.to_host(pin1 + o_hc, d_ctr, sizeof(Counters) * B);
    CK(cudaStreamSynchronize(st));
    memcpy(hc.data(), pin1 + o_hc, sizeof(Counters) * B);
    // ---- allocate the rest from the totals
    bool any_zeroed = false;
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      std::string m;
      lc_status s = counters_status(hc[i], &m);
      if (s != LC_OK) job_fail(r, s, m);
      if (!r.failed && hc[i].n_blocks_in > r.cap_blk)
        job_fail(r, LC_ERR_CORRUPT, "more blocks than bytes allow");
      if (!r.failed && (hc[i].n_entries_in >= (1ull << 32) - 2 || hc[i].key_bytes_in >= (1ull << 32)))
        job_fail(r, LC_ERR_UNSUPPORTED, "more than 2^32 entries or key bytes in one job");
      if (r.failed) {
        // a failed job does no more work: zero counts, no merge children
        hc[i] = Counters{};
        hc[i].error = kErrLimit;
        r.J.n_runs = 0;
        r.J.n_gp = 0;
        any_zeroed = true;
      }
      r.N = r.failed ? 0 : hc[i].n_entries_in;
      if (exact) {
        r.K = r.failed ? 0 : hc[i].key_bytes_in;
        r.max_klen = std::max<uint32_t>(hc[i].max_klen, 8);
      } else {
        r.K = r.failed ? 0 : std::min<uint64_t>(r.in_bytes + 65536, (1ull << 32) - 1);
        r.max_klen = kFastMaxKey;
      }
      r.J.reserve_keys = exact ? 0 : 1;
      r.J.max_key_len = kFastMaxKey;
      // blocks of many entries are walked 8 to a warp (four restart runs of
      // 16 entries each fill its lanes), blocks of few 32
      r.J.dec_group = (!r.failed && hc[i].n_entries_in > 16 * hc[i].n_blocks_in) ? 8 : 32;
      r.j->entries_in = r.N;
      r.j->key_bytes_in = exact ? r.K : 0;
    }
    // (the zeroed counters are uploaded below, from pinned memory)
    uint32_t max_runs = 1;
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      alloc_tail(r, A, true);
      if (r.failed) {
        // run_entry_begin[0] must read 0 for the merge kernels
        CK(cudaMemsetAsync(r.J.run_entry_begin_w, 0, 8, st));
      }
      max_runs = std::max<uint32_t>(max_runs, r.J.n_runs);
      bt.max_entries = std::max<uint64_t>(bt.max_entries, r.N);
      bt.max_gp = std::max<uint32_t>(bt.max_gp, r.J.n_gp);
      bt.max_cap_triggers = std::max<uint32_t>(bt.max_cap_triggers, r.J.cap_triggers);
      bt.max_cap_files = std::max<uint32_t>(bt.max_cap_files, r.J.cap_files);
    }
    // the batch's device memory is now known (every array is sized): the
    // admission charge becomes what the batch holds
    if (admitted) trueup.set((int64_t)A.used - (int64_t)admitted);
    // grid shapes in powers of two, so that batches of similar size share a
    // captured graph (the kernels loop over whatever the grid leaves)
    bt.max_entries = pow2_at_least(std::max<uint64_t>(bt.max_entries, 1));
    bt.max_blocks_in = pow2_at_least(bt.max_blocks_in);  // decode grid size only
    bt.max_cap_files = (uint32_t)pow2_at_least(bt.max_cap_files);
    bt.max_cap_triggers = (uint32_t)pow2_at_least(bt.max_cap_triggers);
    bt.max_gp = bt.max_gp ? (uint32_t)pow2_at_least(bt.max_gp + 1) - 1 : 0;
    bt.merge_rounds = ceil_log2(max_runs);
    bt.max_runs = max_runs;
    // every job's per-file results in one device region, read back with one
    // copy: [files | key offsets | keys] per job
    std::vector<size_t> res_off(B + 1, 0);
    for (uint32_t i = 0; i < B; i++) {
      const JobDev& J = runs[i].J;
      const size_t sz = ((sizeof(FileOut) * J.cap_files + 15) & ~size_t(15)) +
                        ((8 * (2ull * J.cap_files + 1) + 15) & ~size_t(15)) +
                        ((2ull * J.cap_files * runs[i].max_klen + 1 + 15) & ~size_t(15));
      res_off[i + 1] = res_off[i] + sz;
    }
    uint8_t* d_res = A.get<uint8_t>(res_off[B]);
    for (uint32_t i = 0; i < B; i++) {
      JobDev& J = runs[i].J;
      uint8_t* q = d_res + res_off[i];
      J.files = reinterpret_cast<FileOut*>(q);
      q += (sizeof(FileOut) * J.cap_files + 15) & ~size_t(15);
      J.fkoff = reinterpret_cast<uint64_t*>(q);
      q += (8 * (2ull * J.cap_files + 1) + 15) & ~size_t(15);
      J.fkeys = q;
    }
    // pinned staging after the first sync: [counters | descriptors | results]
    const size_t p_hj = (sizeof(Counters) * B + 255) & ~size_t(255);
    const size_t p_res = p_hj + ((sizeof(JobDev) * B + 255) & ~size_t(255));
    uint8_t* pin2 = slot.pinned(p_res + res_off[B]);
    if (any_zeroed) {
      memcpy(pin2, hc.data(), sizeof(Counters) * B);
      slot.to_device(d_ctr, pin2, sizeof(Counters) * B);
    }
    JobDev* hj2 = reinterpret_cast<JobDev*>(pin2 + p_hj);
    for (uint32_t i = 0; i < B; i++) hj2[i] = runs[i].J;
    slot.to_device(slot.d_jobs, (const uint8_t*)hj2, sizeof(JobDev) * B);
    T.start();
    // ---- decode, merge, drop, partition, encode: one graph launch
    const int how = slot.run_tail(bt, true, e->use_graphs, T);
    (how == 0 ? e->n_direct : how == 1 ? e->n_captures : e->n_replays)++;
    e->n_batches++;
    e->n_jobs += B;
    // ---- per-job results: two transfers into pinned memory, one sync
    slot.to_host(pin2 + p_res, d_res, res_off[B]);
    slot.to_host(pin2, d_ctr, sizeof(Counters) * B);
    CK(cudaStreamSynchronize(st));
    memcpy(hc.data(), pin2, sizeof(Counters) * B);
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      const uint8_t* q = pin2 + p_res + res_off[i];
      r.files.resize(r.J.cap_files);
      r.koff.resize(2ull * r.J.cap_files + 1);
      r.j->key_bytes.resize(2ull * r.J.cap_files * r.max_klen + 1);
      const uint32_t nf = std::min<uint32_t>(hc[i].n_files, r.J.cap_files);
      memcpy(r.files.data(), q, sizeof(FileOut) * nf);
      q += (sizeof(FileOut) * r.J.cap_files + 15) & ~size_t(15);
      memcpy(r.koff.data(), q, 8 * (2ull * nf + 1));
      q += (8 * (2ull * r.J.cap_files + 1) + 15) & ~size_t(15);
      // keys in fixed slots of max_klen bytes, their lengths in koff
      const uint64_t kb = 2ull * nf * r.max_klen;
      memcpy(r.j->key_bytes.data(), q, std::min<uint64_t>(kb, r.j->key_bytes.size()));
    }
    std::vector<lc_job*> retry;  // single-pass jobs whose key arena was too small
    // downloads of this batch after the previous batch's (CopyLane)
    std::unique_lock<std::mutex> down_lk(e->down_lane.mu, std::defer_lock);
    bool host_down = false;
    for (uint32_t i = 0; i < B; i++)
      host_down = host_down || (!runs[i].failed && runs[i].j->outputs_on_device != 1 &&
                                hc[i].bytes_out && !hc[i].error);
    if (host_down) {
      down_lk.lock();
      if (e->down_lane.any) CK(cudaStreamWaitEvent(st, e->down_lane.done, 0));
    }
    for (uint32_t i = 0; i < B; i++) {
      JobRun& r = runs[i];
      if (r.failed) continue;
      if (!exact && hc[i].error == kErrRetryExact) {
        retry.push_back(r.j);
        r.failed = true;
        continue;
      }
      if (!exact) r.j->key_bytes_in = hc[i].key_cursor;
      std::string m;
      lc_status s = counters_status(hc[i], &m);
      if (s != LC_OK) {
        job_fail(r, s, m);
        continue;
      }
      lc_job* j = r.j;
      const uint64_t nbytes = hc[i].bytes_out;
      if (j->outputs_on_device != 1 && nbytes) {
        j->h_out = e->pinned.take(nbytes, &j->h_out_cap);
        if (!j->h_out) {
          job_fail(r, LC_ERR_NO_MEMORY, "pinned host buffer");
          continue;
        }
        copy_pieces(j->h_out, r.J.out, nbytes, cudaMemcpyDeviceToHost, st, piece_for(nbytes));
      }
      const uint32_t nf = hc[i].n_files;
      j->file_offset.resize(nf);
      j->file_size.resize(nf);
      j->file_entries.resize(nf);
      j->small_off.resize(nf);
      j->large_off.resize(nf);
      j->small_len.resize(nf);
      j->large_len.resize(nf);
      for (uint32_t f = 0; f < nf; f++) {
        const FileOut& F = r.files[f];
        j->file_offset[f] = F.out_off;
        j->file_size[f] = F.size;
        j->file_entries[f] = F.end_kept - F.first_kept;
        j->small_off[f] = 2ull * f * r.max_klen;
        j->small_len[f] = (uint32_t)r.koff[2 * f];
        j->large_off[f] = (2ull * f + 1) * r.max_klen;
        j->large_len[f] = (uint32_t)r.koff[2 * f + 1];
      }
      j->bytes_out = nbytes;
      j->entries_out = hc[i].n_kept;
      j->kept_key_bytes = hc[i].kept_key_bytes;
      j->kept_value_bytes = hc[i].kept_value_bytes;
      if (j->outputs_on_device == 1 || j->outputs_on_device == 2) j->d_out = r.J.out;
      if (r.J.dec_keys) {
        // every output file's decoded entries: views into the job's buffer
        j->d_dec = r.dec_block;
        j->d_dec_cap = r.dec_cap;
        j->out_dec.resize(nf);
        j->out_dec_ptrs.resize(nf);
        for (uint32_t f = 0; f < nf; f++) {
          const uint64_t k0 = r.files[f].first_kept;
          lc_decoded& x = j->out_dec[f];
          x.run.n = r.files[f].end_kept - k0;
          x.run.keys = r.J.dec_keys;
          x.run.kcum = r.J.dec_kcum + k0;
          x.run.vlen = r.J.dec_vlen + k0;
          x.run.vpos = r.J.dec_vpos + k0;
          x.run.pfx = r.J.dec_pfx + k0;
          x.run.tag = r.J.dec_tag + k0;
          x.table_size = r.files[f].size;
          j->out_dec_ptrs[f] = &x;
        }
      }
    }
    if (host_down) {
      CK(cudaEventRecord(e->down_lane.done, st));
      e->down_lane.any = true;
      down_lk.unlock();
    }
    T.mark(kDownload);
    CK(cudaEventRecord(ev1, st));
    CK(cudaStreamSynchronize(st));
    // outputs kept on the device hold their bytes only (the capacity was a
    // bound taken before the layout was known)
    for (uint32_t i = 0; i < B; i++)
      if (jobs[i]->d_out) jobs[i]->d_out_cap = A.trim(jobs[i]->d_out, jobs[i]->bytes_out);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    std::vector<float> ph;
    T.collect(ph);
    const uint32_t launches = launches_on_this_thread() - launches0;
    std::vector<void*> keep;
    for (uint32_t i = 0; i < B; i++) {
      lc_job* j = jobs[i];
      j->device_ms = ms;
      j->phase_ms = ph;
      j->launches = launches;
      j->batch_jobs = B;
      if (!runs[i].failed) j->status = LC_OK;
      if (j->d_out) keep.push_back(j->d_out);
      if (j->d_dec) keep.push_back(j->d_dec);
    }
    A.release(keep);  // the batch has completed: its scratch serves the next one at once
    if (!retry.empty()) {
      cudaEventDestroy(ev0);
      cudaEventDestroy(ev1);
      e->n_exact_reruns += retry.size();
      // this batch's scratch is released: the rerun holds the charge
      trueup.set(0);
      uint64_t readmit = 0;
      if (admitted)
        for (auto* j : retry) readmit += j->est_bytes;
      run_batch(retry, slot, tun, true, readmit);
      return;
    }
  } catch (const CudaError& ce) {
    cudaStreamSynchronize(st);
    A.release({});
    for (auto* j : jobs) {
      j->d_out = nullptr;
      j->d_dec = nullptr;
      j->out_dec_ptrs.clear();
      j->status = LC_ERR_CUDA;
      j->err = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
    }
  } catch (const StatusError& se) {
    cudaStreamSynchronize(st);
    A.release({});
    for (auto* j : jobs) {
      j->d_out = nullptr;
      j->d_dec = nullptr;
      j->out_dec_ptrs.clear();
      j->status = se.s;
      j->err = se.msg;
    }
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
}

// Flush encoder: one table from sorted entries (kind 1), a batch of one that
// skips decode, merge and the drop rule.
void run_build(lc_job* j, lc_slot& slot) {
  lc_engine* e = j->eng;
  cudaStream_t st = slot.st;
  DevAlloc A(st, e);
  PhaseTimer T((e->flags & LC_FLAG_PHASE_TIMING) != 0, st);
  const uint32_t launches0 = launches_on_this_thread();
  try {
    T.start();
    JobRun r;
    r.j = j;
    fill_common(r.J, j, e);
    JobDev& J = r.J;
    J.max_file_size = ~0ull;  // BuildTable writes one file
    J.max_gp_overlap = 0;
    const uint64_t N = (uint64_t)j->bn;
    std::vector<uint64_t> hk;
    const uint64_t* ko = j->bkoffs;
    uint64_t vb;
    if (j->inputs_on_device) {
      hk.resize(N + 1);
      CK(cudaMemcpyAsync(hk.data(), j->bkoffs, (N + 1) * 8, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&vb, j->bvoffs + N, 8, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      ko = hk.data();
    } else {
      vb = j->bvoffs[N];
    }
    const uint64_t kb = ko[N];
    if (kb >= (1ull << 32) || vb >= (1ull << 32) || N >= (1ull << 32) - 2)
      throw StatusError{LC_ERR_UNSUPPORTED, "table input beyond 4 GiB"};
    for (uint64_t i = 0; i < N; i++)
      r.max_klen = std::max<uint32_t>(r.max_klen, (uint32_t)(ko[i + 1] - ko[i]));
    const cudaMemcpyKind kind = j->inputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    J.keys = A.get<uint8_t>(kb + 16);
    uint8_t* d_vals = A.get<uint8_t>(vb + 16);
    uint64_t* d_ko = A.get<uint64_t>(N + 1);
    uint64_t* d_vo = A.get<uint64_t>(N + 1);
    if (kb) copy_pieces(J.keys, j->bkeys, kb, kind, st, piece_for(kb + vb));
    if (vb) copy_pieces(d_vals, j->bvals, vb, kind, st, piece_for(kb + vb));
    CK(cudaMemcpyAsync(d_ko, j->bkoffs, (N + 1) * 8, kind, st));
    CK(cudaMemcpyAsync(d_vo, j->bvoffs, (N + 1) * 8, kind, st));
    J.in = d_vals;
    J.in_size = vb;
    r.in_bytes = vb;
    J.in_end = d_vals + vb + 16;
    J.src_koffs = d_ko;
    J.src_voffs = d_vo;
    J.cap_key_bytes = kb;
    J.cap_entries = N;
    J.ctr = A.get<Counters>(1);
    Counters init{};
    init.n_kept = N;
    init.n_entries_in = N;
    CK(cudaMemcpyAsync(J.ctr, &init, sizeof(Counters), cudaMemcpyHostToDevice, st));
    J.e_koff = A.get<uint32_t>(N);
    J.e_klen = A.get<uint32_t>(N);
    J.e_voff = A.get<uint32_t>(N);
    J.e_vlen = A.get<uint32_t>(N);
    J.e_pfx = A.get<uint64_t>(N);
    J.e_tag = A.get<uint64_t>(N);
    J.k_forced = A.get<uint8_t>(N + 1);
    CK(cudaMemsetAsync(J.k_forced, 0, N + 1, st));
    J.kept_pos = A.get<uint32_t>(N + 1);
    r.N = N;
    r.K = kb;
    alloc_tail(r, A, false);
    CK(cudaMemcpyAsync(slot.d_jobs, &J, sizeof(JobDev), cudaMemcpyHostToDevice, st));
    Batch bt;
    bt.d = slot.d_jobs;
    bt.B = 1;
    bt.max_entries = std::max<uint64_t>(N, 1);
    bt.max_cap_files = J.cap_files;
    bt.max_cap_triggers = J.cap_triggers;
    T.mark(kUpload);
    launch_entries_from_offsets(bt, st);
    CK(cudaGetLastError());
    launch_tail(bt, false, st, T);
    CK(cudaGetLastError());
    Counters hc;
    r.files.resize(J.cap_files);
    r.koff.resize(2ull * J.cap_files + 1);
    j->key_bytes.resize(2ull * J.cap_files * r.max_klen + 1);
    CK(cudaMemcpyAsync(&hc, J.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(r.files.data(), J.files, J.cap_files * sizeof(FileOut), cudaMemcpyDeviceToHost,
                       st));
    CK(cudaMemcpyAsync(r.koff.data(), J.fkoff, r.koff.size() * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(j->key_bytes.data(), J.fkeys, j->key_bytes.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::string m;
    lc_status s = counters_status(hc, &m);
    if (s != LC_OK) throw StatusError{s, m};
    const uint64_t nbytes = hc.bytes_out;
    if (nbytes) {
      j->h_out = e->pinned.take(nbytes, &j->h_out_cap);
      if (!j->h_out) throw StatusError{LC_ERR_NO_MEMORY, "pinned host buffer"};
      copy_pieces(j->h_out, J.out, nbytes, cudaMemcpyDeviceToHost, st, piece_for(nbytes));
    }
    const uint32_t nf = hc.n_files;
    j->file_offset.resize(nf);
    j->file_size.resize(nf);
    j->file_entries.resize(nf);
    j->small_off.resize(nf);
    j->large_off.resize(nf);
    j->small_len.resize(nf);
    j->large_len.resize(nf);
    for (uint32_t f = 0; f < nf; f++) {
      j->file_offset[f] = r.files[f].out_off;
      j->file_size[f] = r.files[f].size;
      j->file_entries[f] = r.files[f].end_kept - r.files[f].first_kept;
      j->small_off[f] = 2ull * f * r.max_klen;
      j->small_len[f] = (uint32_t)r.koff[2 * f];
      j->large_off[f] = (2ull * f + 1) * r.max_klen;
      j->large_len[f] = (uint32_t)r.koff[2 * f + 1];
    }
    T.mark(kDownload);
    CK(cudaStreamSynchronize(st));
    j->entries_in = N;
    j->key_bytes_in = kb;
    j->bytes_out = nbytes;
    j->entries_out = hc.n_kept;
    j->kept_key_bytes = hc.kept_key_bytes;
    j->kept_value_bytes = hc.kept_value_bytes;
    T.collect(j->phase_ms);
    j->launches = launches_on_this_thread() - launches0;
    j->status = LC_OK;
    A.release({});
    CK(cudaStreamSynchronize(st));
  } catch (const CudaError& ce) {
    cudaStreamSynchronize(st);
    A.release({});
    j->status = LC_ERR_CUDA;
    j->err = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
  } catch (const StatusError& se) {
    cudaStreamSynchronize(st);
    A.release({});
    j->status = se.s;
    j->err = se.msg;
  }
}

// Device bytes a job is admitted with, from the sizes run_batch gives its
// arrays: the input copy (host inputs), the per-block parse arrays, the key
// arena, the output and the per-entry arrays.  The entry count is not known
// before the parse; it is taken as one entry per kEstEntryBytes of input
// (the at-size workloads have 67-250 bytes per entry) and the worker trues
// the charge up to the batch's real allocation once the counts are known.
constexpr uint64_t kEstEntryBytes = 40;
constexpr uint64_t kEntryArrayBytes = 248;  // per-entry arrays of alloc_tail, rounded up
uint64_t estimate_bytes(const lc_job* j) {
  uint64_t in = 0;
  for (auto& t : j->tables) in += round16(t.size);
  if (j->kind == 1) in = j->bkoffs ? j->bkoffs[j->bn] + j->bvoffs[j->bn] : 0;
  const uint64_t n_est = in / kEstEntryBytes + 1;
  const uint64_t host_copy = j->inputs_on_device ? 0 : in + 16;
  const uint64_t parse = (in / 13 + j->tables.size() + 1) * 48;
  const uint64_t arena = in + 65536;
  const uint64_t out = in + in / 4 + n_est * 66 + 65536;
  const uint64_t dec = j->keep_decoded ? arena + n_est * 32 : 0;
  return host_copy + parse + arena + out + dec + n_est * kEntryArrayBytes + (8ull << 20);
}

void finish(lc_job* j) {
  lc_engine* e = j->eng;
  {
    std::lock_guard<std::mutex> g(j->mu);
    j->done = true;
    j->cv.notify_all();
  }
  std::lock_guard<std::mutex> g(e->done_mu);
  e->done_cv.notify_all();
}

bool job_done(lc_job* j) {
  std::lock_guard<std::mutex> g(j->mu);
  return j->done;
}

// Worker: takes the head of the queue plus every further queued job that
// still fits the device budget (up to max_batch) and runs them as one batch.
// Jobs that arrive while a batch is on the device join the next one.
void worker_main(lc_engine* e, lc_slot* wslot) {
  lc_slot& slot = *wslot;
  while (true) {
    std::vector<lc_job*> batch;
    uint64_t bytes = 0, in_bytes = 0;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv.wait(lk, [&] { return e->stop || !e->queue.empty(); });
      if (e->stop && e->queue.empty()) break;
      lc_job* head = e->queue.front();
      e->admit_cv.wait(lk, [&] {
        return e->stop || e->inflight_bytes == 0 || e->inflight_bytes + head->est_bytes <= e->budget;
      });
      if (e->queue.empty() || e->queue.front() != head) continue;
      while (!e->queue.empty() && batch.size() < e->max_batch) {
        lc_job* j = e->queue.front();
        if (j->kind != 0) {
          if (batch.empty()) {
            batch.push_back(j);
            bytes += j->est_bytes;
            e->queue.pop_front();
          }
          break;
        }
        if (!batch.empty() && (e->inflight_bytes + bytes + j->est_bytes > e->budget ||
                               in_bytes + j->bytes_in > e->max_batch_bytes))
          break;
        batch.push_back(j);
        bytes += j->est_bytes;
        in_bytes += j->bytes_in;
        e->queue.pop_front();
      }
      e->inflight_bytes += bytes;
    }
    const auto t_start = std::chrono::steady_clock::now();
    for (auto* j : batch)
      j->queue_ms = std::chrono::duration<double, std::milli>(t_start - j->t_submit).count();
    if (e->stop) {
      for (auto* j : batch) j->status = LC_ERR_SHUTDOWN;
    } else {
      cudaSetDevice(e->device);
      if (batch.size() == 1 && batch[0]->kind == 1) run_build(batch[0], slot);
      else run_batch(batch, slot, e->tuning(), false, bytes);
    }
    {
      std::lock_guard<std::mutex> g(e->mu);
      e->inflight_bytes -= bytes;
    }
    e->admit_cv.notify_all();
    e->cv.notify_all();
    for (auto* j : batch) finish(j);
  }
}

lc_status fail(lc_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

lc_status copy_desc(lc_job* j, const lc_job_desc* d) {
  if (d->n_tables < 0 || d->n_runs < 0 || (d->n_tables > 0 && !d->tables) ||
      (d->n_runs > 0 && !d->run_table_count))
    return fail(LC_ERR_INVALID_ARG, "bad table or run arrays");
  int64_t sum = 0;
  for (int i = 0; i < d->n_runs; i++) {
    if (d->run_table_count[i] <= 0) return fail(LC_ERR_INVALID_ARG, "empty merge child");
    sum += d->run_table_count[i];
  }
  if (sum != d->n_tables) return fail(LC_ERR_INVALID_ARG, "run table counts do not sum to n_tables");
  if (d->options.block_size == 0 || d->options.restart_interval == 0 ||
      d->options.max_file_size == 0)
    return fail(LC_ERR_INVALID_ARG, "zero block size, restart interval or max file size");
  j->level = d->level;
  j->tables.assign(d->tables, d->tables + d->n_tables);
  for (auto& t : j->tables)
    if (t.size && !t.data) return fail(LC_ERR_INVALID_ARG, "table without data");
  j->run_counts.assign(d->run_table_count, d->run_table_count + d->n_runs);
  for (int i = 0; i < d->n_grandparents; i++) {
    const lc_file_range& g = d->grandparents[i];
    if (g.largest_len < 8) return fail(LC_ERR_INVALID_ARG, "grandparent key shorter than 8 bytes");
    j->gp_largest.emplace_back((const char*)g.largest, g.largest_len);
    j->gp_size.push_back(g.file_size);
  }
  for (int i = 0; i < d->n_base_files; i++) {
    const lc_file_range& f = d->base_files[i];
    if (f.smallest_len < 8 || f.largest_len < 8)
      return fail(LC_ERR_INVALID_ARG, "base-level key shorter than 8 bytes");
    if (i > 0 && f.level < d->base_files[i - 1].level)
      return fail(LC_ERR_INVALID_ARG, "base-level files must be grouped by level");
    j->base_level.push_back(f.level);
    j->base_small.emplace_back((const char*)f.smallest, f.smallest_len - 8);
    j->base_large.emplace_back((const char*)f.largest, f.largest_len - 8);
  }
  j->smallest_snapshot = d->smallest_snapshot;
  j->opt = d->options;
  j->inputs_on_device = d->inputs_on_device;
  if (d->outputs_on_device < 0 || d->outputs_on_device > 2)
    return fail(LC_ERR_INVALID_ARG, "outputs_on_device must be 0, 1 or 2");
  j->outputs_on_device = d->outputs_on_device;
  j->verify_checksums = d->verify_checksums;
  if (d->keep_decoded && d->outputs_on_device != 1 && d->outputs_on_device != 2)
    return fail(LC_ERR_INVALID_ARG, "keep_decoded needs outputs kept on the device");
  j->keep_decoded = d->keep_decoded ? 1 : 0;
  if (d->decoded) {
    j->in_dec.assign(d->decoded, d->decoded + d->n_tables);
    for (int32_t t = 0; t < d->n_tables; t++) {
      const lc_decoded* x = d->decoded[t];
      if (!x) continue;
      if (!d->inputs_on_device)
        return fail(LC_ERR_INVALID_ARG, "a decoded table must be read from device memory");
      if (x->table_size != d->tables[t].size)
        return fail(LC_ERR_INVALID_ARG, "decoded form of another table (size differs)");
      j->decoded_inputs++;
    }
  }
  for (auto& t : j->tables) j->bytes_in += t.size;
  return LC_OK;
}

void fill_out(lc_job* j, lc_job_out* o) {
  memset(o, 0, sizeof(*o));
  o->n_files = (int32_t)j->file_size.size();
  o->data = j->outputs_on_device == 1 ? j->d_out : j->h_out;
  o->file_offset = j->file_offset.data();
  o->file_size = j->file_size.data();
  o->file_entries = j->file_entries.data();
  o->key_bytes = j->key_bytes.data();
  o->smallest_offset = j->small_off.data();
  o->smallest_len = j->small_len.data();
  o->largest_offset = j->large_off.data();
  o->largest_len = j->large_len.data();
  o->bytes_in = j->bytes_in;
  o->bytes_out = j->bytes_out;
  o->entries_in = j->entries_in;
  o->entries_out = j->entries_out;
  o->device_ms = j->device_ms;
  o->kernel_launches = j->launches;
  o->n_phases = j->phase_ms.empty() ? 0 : (uint32_t)j->phase_ms.size();
  o->phase_name = kPhaseNames;
  o->phase_ms = j->phase_ms.data();
  o->key_bytes_in = j->key_bytes_in;
  o->value_bytes_out = j->kept_value_bytes;
  o->key_bytes_out = j->kept_key_bytes;
  o->device_data = j->d_out;
  o->batch_jobs = j->batch_jobs;
  o->queue_ms = j->queue_ms;
  o->decoded = j->keep_decoded && !j->out_dec_ptrs.empty() ? j->out_dec_ptrs.data() : nullptr;
  o->decoded_inputs = j->decoded_inputs;
}

// The engine's CRC tables, one device array: [x^(8n) | row fields | x^(-8n) |
// byte table | all-ones shifts | long shifts].
//  * x^(8n) mod P for n < kCrcXpowN (register shifts by n zero bytes);
//  * for the row CRC: entry kCrcFieldEntries i + v is the register after 16
//    bytes holding v at bits [W i, W i + W) (W = kCrcFieldBits) and zero
//    elsewhere, then kCrcRowBytes - 16 zero bytes, from register 0;
//  * x^(-8n) mod P for n < kCrcXinvN: the shift that undoes n zero bytes;
//  * the byte table: the register after byte i, from 0;
//  * for n < kCrcXpowN, the register after n zero bytes from all ones (the
//    CRC's initial register carried to the end of an n-byte message);
//  * x^(8 kCrcXpowN h) mod P for h < kCrcXpowN: with the first table, any
//    shift below kCrcXpowN^2 bytes is one product of two entries.
// Registers are reflected (bit 31 is x^0), as in util/crc32c.cc.
uint32_t host_crc_byte(uint32_t c, uint8_t b) {
  c ^= b;
  for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
  return c;
}

void host_crc_tables(std::vector<uint32_t>& t) {
  t.assign(kCrcXpowN + kCrcH5Words + kCrcXinvN + 256 + 2 * kCrcXpowN, 0);
  uint32_t c = 0x80000000u;  // x^0
  for (uint32_t m = 0; m < kCrcXpowN; m++) {
    t[m] = c;
    c = host_crc_byte(c, 0);
  }
  uint32_t* h5 = t.data() + kCrcXpowN;
  for (uint32_t i = 0; i < kCrcFields; i++)
    for (uint32_t v = 0; v < kCrcFieldEntries; v++) {
      uint8_t x[16] = {};
      for (uint32_t bit = 0; bit < kCrcFieldBits; bit++) {
        const uint32_t at = kCrcFieldBits * i + bit;
        if (((v >> bit) & 1) && at < 128) x[at >> 3] |= (uint8_t)(1u << (at & 7));
      }
      uint32_t r = 0;
      for (uint32_t k = 0; k < 16; k++) r = host_crc_byte(r, x[k]);
      for (uint32_t k = 16; k < kCrcRowBytes; k++) r = host_crc_byte(r, 0);
      h5[kCrcFieldEntries * i + v] = r;
    }
  // one zero byte maps c to byte(c & 0xff) ^ (c >> 8), where byte(i) =
  // host_crc_byte(0, i): its top byte names i (the table's top bytes are a
  // permutation), which undoes the step
  uint32_t by_top[256];
  for (uint32_t i = 0; i < 256; i++) by_top[host_crc_byte(0, (uint8_t)i) >> 24] = i;
  uint32_t* xinv = h5 + kCrcH5Words;
  c = 0x80000000u;
  for (uint32_t n = 0; n < kCrcXinvN; n++) {
    xinv[n] = c;
    const uint32_t i = by_top[c >> 24];
    c = ((c ^ host_crc_byte(0, (uint8_t)i)) << 8) | i;
  }
  uint32_t* byte = xinv + kCrcXinvN;
  for (uint32_t i = 0; i < 256; i++) byte[i] = host_crc_byte(0, (uint8_t)i);
  uint32_t* ones = byte + 256;
  c = 0xffffffffu;
  for (uint32_t n = 0; n < kCrcXpowN; n++) {
    ones[n] = c;
    c = host_crc_byte(c, 0);
  }
  uint32_t* hi = ones + kCrcXpowN;
  const uint32_t step = gf2_mulmod(t[kCrcXpowN - 1], t[1]);  // x^(8 kCrcXpowN)
  c = 0x80000000u;
  for (uint32_t h = 0; h < kCrcXpowN; h++) {
    hi[h] = c;
    c = gf2_mulmod(c, step);
  }
}

}  // namespace

extern "C" {

const char* lc_version(void) { return kVersion; }
const char* lc_last_error(void) { return g_last_error.c_str(); }
}  // extern "C"

// The error text of entry points outside this file (lc_noalloc.cu).
void lc::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

const char* lc_status_string(lc_status s) {
  switch (s) {
    case LC_OK: return "ok";
    case LC_ERR_INVALID_ARG: return "invalid argument";
    case LC_ERR_CORRUPT: return "corruption";
    case LC_ERR_CUDA: return "cuda error";
    case LC_ERR_NO_MEMORY: return "out of memory";
    case LC_ERR_BUDGET: return "over device budget";
    case LC_ERR_TIMEOUT: return "timeout";
    case LC_ERR_UNSUPPORTED: return "unsupported";
    case LC_ERR_SHUTDOWN: return "shutting down";
  }
  return "unknown";
}

lc_status lc_engine_create(const lc_config* cfg, lc_engine** out) {
  if (!out) return fail(LC_ERR_INVALID_ARG, "null engine pointer");
  lc_engine* e = new (std::nothrow) lc_engine();
  if (!e) return fail(LC_ERR_NO_MEMORY, "engine");
  uint64_t pinned_reserve = 0;
  if (cfg) {
    e->device = cfg->device;
    if (cfg->device_budget_bytes) e->budget = cfg->device_budget_bytes;
    if (cfg->max_inflight_jobs > 0) e->max_inflight = cfg->max_inflight_jobs;
    if (cfg->max_batch_jobs > 0) e->max_batch = (uint32_t)cfg->max_batch_jobs;
    if (cfg->max_batch_bytes) e->max_batch_bytes = cfg->max_batch_bytes;
    pinned_reserve = cfg->pinned_reserve_bytes;
    e->flags = cfg->flags;
    e->use_graphs = (cfg->flags & LC_FLAG_NO_GRAPHS) == 0;
  }
  std::vector<lc_slot*> wslots;
  try {
    CK(cudaSetDevice(e->device));
    if (pinned_reserve && !e->pinned.add_slab(pinned_reserve))
      throw CudaError{cudaErrorMemoryAllocation, "cudaMallocHost (pinned_reserve_bytes)"};
    // the pool keeps freed memory for reuse across jobs (trimming it at every
    // synchronisation costs milliseconds per job) up to three quarters of the
    // device; beyond that it is returned at synchronisation points, so that
    // allocations of many different sizes cannot grow it without bound
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, e->device));
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    uint64_t thr = std::max<uint64_t>(e->budget, total_b / 4 * 3);
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    decode_kernel_attributes();
    encode_kernel_attributes();
    merge_kernel_attributes();
    CK(cudaGetLastError());
    std::vector<uint32_t> t;
    host_crc_tables(t);
    CK(cudaMalloc(&e->crc_xpow, t.size() * 4));
    CK(cudaMemcpy(e->crc_xpow, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaEventCreateWithFlags(&e->up_lane.done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&e->down_lane.done, cudaEventDisableTiming));
    for (int i = 0; i < e->max_inflight; i++) {
      std::unique_ptr<lc_slot> sl(new lc_slot());
      sl->init(e->device, e->max_batch);
      sl->grow_count = &e->n_staging_grows;
      wslots.push_back(sl.get());
      e->slots.push_back(std::move(sl));
    }
  } catch (const CudaError& ce) {
    std::string m = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
    if (e->crc_xpow) cudaFree(e->crc_xpow);
    if (e->up_lane.done) cudaEventDestroy(e->up_lane.done);
    if (e->down_lane.done) cudaEventDestroy(e->down_lane.done);
    e->dev_out.clear();
    e->scratch.clear();
    e->pinned.clear();
    delete e;
    return fail(LC_ERR_CUDA, m);
  }
  for (lc_slot* sl : wslots) e->workers.emplace_back(worker_main, e, sl);
  *out = e;
  return LC_OK;
}

void lc_engine_destroy(lc_engine* e) {
  if (!e) return;
  {
    std::lock_guard<std::mutex> g(e->mu);
    e->stop = true;
  }
  e->cv.notify_all();
  e->admit_cv.notify_all();
  for (auto& w : e->workers) w.join();
  cudaSetDevice(e->device);
  e->pinned.clear();
  e->dev_out.clear();
  e->scratch.clear();
  cudaFree(e->crc_xpow);
  cudaEventDestroy(e->up_lane.done);
  cudaEventDestroy(e->down_lane.done);
  delete e;  // destroys the slots
}

lc_status lc_job_submit(lc_engine* e, const lc_job_desc* desc, lc_job** out) {
  if (!e || !desc || !out) return fail(LC_ERR_INVALID_ARG, "null argument");
  lc_job* j = new (std::nothrow) lc_job();
  if (!j) return fail(LC_ERR_NO_MEMORY, "job");
  j->eng = e;
  lc_status s = copy_desc(j, desc);
  if (s != LC_OK) {
    delete j;
    return s;
  }
  j->est_bytes = estimate_bytes(j);
  if (j->est_bytes > e->budget) {
    delete j;
    return fail(LC_ERR_BUDGET, "job needs more device memory than the engine budget");
  }
  {
    std::lock_guard<std::mutex> g(e->mu);
    if (e->stop) {
      delete j;
      return fail(LC_ERR_SHUTDOWN, "engine stopping");
    }
    j->t_submit = std::chrono::steady_clock::now();
    e->queue.push_back(j);
  }
  e->cv.notify_one();
  *out = j;
  return LC_OK;
}

lc_status lc_estimate_device_bytes(const lc_job_desc* desc, uint64_t* bytes) {
  if (!desc || !bytes) return fail(LC_ERR_INVALID_ARG, "null argument");
  lc_job j;
  lc_status s = copy_desc(&j, desc);
  if (s != LC_OK) return s;
  *bytes = estimate_bytes(&j);
  return LC_OK;
}

lc_status lc_job_wait(lc_job* j, int64_t timeout_ns) {
  if (!j) return fail(LC_ERR_INVALID_ARG, "null job");
  std::unique_lock<std::mutex> lk(j->mu);
  if (timeout_ns < 0) {
    j->cv.wait(lk, [&] { return j->done; });
  } else if (!j->cv.wait_for(lk, std::chrono::nanoseconds(timeout_ns), [&] { return j->done; })) {
    return LC_ERR_TIMEOUT;
  }
  if (j->status != LC_OK) g_last_error = j->err;
  return j->status;
}

lc_status lc_job_wait_any(lc_engine* e, lc_job* const* jobs, int32_t n, int64_t timeout_ns,
                          int32_t* index) {
  if (!e || !index || n <= 0 || !jobs) return fail(LC_ERR_INVALID_ARG, "null argument");
  for (int32_t i = 0; i < n; i++)
    if (!jobs[i] || jobs[i]->eng != e) return fail(LC_ERR_INVALID_ARG, "job of another engine");
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(
                                                                 timeout_ns < 0 ? 0 : timeout_ns);
  std::unique_lock<std::mutex> lk(e->done_mu);
  while (true) {
    // finish() notifies under done_mu, so no completion is missed between
    // this check and the wait
    for (int32_t i = 0; i < n; i++)
      if (job_done(jobs[i])) {
        *index = i;
        return LC_OK;
      }
    if (timeout_ns < 0) {
      e->done_cv.wait(lk);
    } else if (e->done_cv.wait_until(lk, deadline) == std::cv_status::timeout) {
      for (int32_t i = 0; i < n; i++)
        if (job_done(jobs[i])) {
          *index = i;
          return LC_OK;
        }
      return LC_ERR_TIMEOUT;
    }
  }
}

lc_status lc_job_result(lc_job* j, lc_job_out* out) {
  if (!j || !out) return fail(LC_ERR_INVALID_ARG, "null argument");
  {
    std::lock_guard<std::mutex> g(j->mu);
    if (!j->done) return fail(LC_ERR_INVALID_ARG, "job not finished");
  }
  if (j->status != LC_OK) return fail(j->status, j->err);
  fill_out(j, out);
  return LC_OK;
}

void lc_job_release(lc_job* j) {
  if (!j) return;
  if (j->h_out) j->eng->pinned.give(j->h_out, j->h_out_cap);
  // the job has completed and the caller has finished reading its output
  if (j->d_out) j->eng->dev_out.give(j->d_out, j->d_out_cap);
  if (j->d_dec) j->eng->dev_out.give(j->d_dec, j->d_dec_cap);
  delete j;
}

lc_status lc_compact(lc_engine* e, const lc_job_desc* desc, lc_job_out* out, lc_job** job_out) {
  if (!e || !desc || !out || !job_out) return fail(LC_ERR_INVALID_ARG, "null argument");
  *job_out = nullptr;
  lc_job* j = nullptr;
  lc_status s = lc_compact_batch(e, 1, desc, &j);
  if (!j) return s;
  if (s != LC_OK) {
    lc_job_release(j);
    return s;
  }
  fill_out(j, out);
  *job_out = j;
  return LC_OK;
}

lc_status lc_compact_batch(lc_engine* e, int32_t n, const lc_job_desc* descs, lc_job** jobs) {
  if (!e || n < 0 || (n && (!descs || !jobs))) return fail(LC_ERR_INVALID_ARG, "null argument");
  std::vector<lc_job*> all(n, nullptr);
  for (int32_t i = 0; i < n; i++) {
    lc_job* j = new (std::nothrow) lc_job();
    lc_status s = j ? copy_desc(j, &descs[i]) : fail(LC_ERR_NO_MEMORY, "job");
    if (j) j->eng = e;
    if (s != LC_OK) {
      const std::string m = g_last_error;
      delete j;
      for (int32_t k = 0; k < i; k++) delete all[k];
      return fail(s, "job " + std::to_string(i) + ": " + m);
    }
    all[i] = j;
  }
  const Tunables tun = e->tuning();
  // Parts of the batch, in order, at most max_batch jobs each.  Inputs in
  // host memory beyond kSplitBytes in all are cut into about kSplitParts
  // parts run on kSplitThreads slots at once, so that one part's upload
  // overlaps another's kernels and a third's download (one batch would do
  // the three in turn: 64 jobs of 606 MB in all ran at 16 GiB/s as one batch,
  // 25-26 GiB/s in 4-12 parts on 3-4 slots, on B200 over PCIe 5).
  constexpr uint64_t kSplitBytes = 128ull << 20;
  constexpr uint64_t kSplitParts = 8;
  constexpr size_t kSplitThreads = 4;
  uint64_t host_bytes = 0;
  for (auto* j : all)
    if (!j->inputs_on_device) host_bytes += j->bytes_in;
  const uint64_t part_bytes =
      host_bytes > kSplitBytes ? std::max<uint64_t>(host_bytes / kSplitParts, 32ull << 20) : ~0ull;
  std::vector<std::vector<lc_job*>> parts;
  uint64_t in_part = 0;
  for (auto* j : all) {
    if (parts.empty() || parts.back().size() >= e->max_batch ||
        (!parts.back().empty() && in_part + j->bytes_in > part_bytes)) {
      parts.emplace_back();
      in_part = 0;
    }
    parts.back().push_back(j);
    in_part += j->bytes_in;
  }
  std::atomic<size_t> next{0};
  std::mutex err_mu;
  std::string cuda_err;
  auto run_parts = [&]() {
    lc_slot* slot = nullptr;
    try {
      CK(cudaSetDevice(e->device));
      slot = e->take_slot();
    } catch (const CudaError& ce) {
      std::lock_guard<std::mutex> g(err_mu);
      cuda_err = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
      return;
    }
    for (size_t k; (k = next++) < parts.size();) {
      try {
        run_batch(parts[k], *slot, tun);
      } catch (const std::exception& ex) {  // host allocation failures
        for (auto* j : parts[k]) {
          j->status = LC_ERR_NO_MEMORY;
          j->err = ex.what();
        }
      }
    }
    e->put_slot(slot);
  };
  const size_t n_threads = part_bytes == ~0ull ? 1 : std::min<size_t>(parts.size(), kSplitThreads);
  std::vector<std::thread> helpers;
  for (size_t t = 1; t < n_threads; t++) helpers.emplace_back(run_parts);
  run_parts();
  for (auto& h : helpers) h.join();
  if (next.load() < parts.size()) {
    // no thread got a slot: nothing ran
    for (auto* j : all) delete j;
    return fail(LC_ERR_CUDA, cuda_err);
  }
  lc_status first = LC_OK;
  for (int32_t i = 0; i < n; i++) {
    all[i]->done = true;
    if (first == LC_OK && all[i]->status != LC_OK) {
      first = all[i]->status;
      g_last_error = "job " + std::to_string(i) + ": " + all[i]->err;
    }
    jobs[i] = all[i];
  }
  return first;
}

lc_status lc_engine_get_stats(lc_engine* e, lc_engine_stats* out) {
  if (!e || !out) return fail(LC_ERR_INVALID_ARG, "null argument");
  memset(out, 0, sizeof(*out));
  out->batches = e->n_batches;
  out->jobs = e->n_jobs;
  out->graph_captures = e->n_captures;
  out->graph_replays = e->n_replays;
  out->direct_tails = e->n_direct;
  out->block_takes = e->n_block_takes;
  out->block_take_us = e->block_take_ns / 1000;
  out->staging_grows = e->n_staging_grows;
  out->pinned_slab_grows = e->pinned.grows;
  out->setup_us_max = e->setup_ns_max / 1000;
  out->exact_reruns = e->n_exact_reruns;
  auto slabs = [](SlabCache& c, uint64_t* total, uint64_t* free_b, uint64_t* peak, uint64_t* grows) {
    std::lock_guard<std::mutex> g(c.mu);
    *total = c.total;
    *peak = c.peak;
    *grows = c.grows;
    for (auto& b : c.free_blocks) *free_b += b.second;
  };
  slabs(e->scratch, &out->scratch_bytes, &out->scratch_free_bytes, &out->scratch_peak_bytes,
        &out->scratch_slab_grows);
  slabs(e->dev_out, &out->device_out_bytes, &out->device_out_free_bytes, &out->device_out_peak_bytes,
        &out->device_out_slab_grows);
  {
    std::lock_guard<std::mutex> g(e->pinned.mu);
    out->pinned_bytes = e->pinned.total;
    for (auto& b : e->pinned.free_blocks) out->pinned_free_bytes += b.second;
  }
  {
    std::lock_guard<std::mutex> g(e->mu);
    out->inflight_bytes = e->inflight_bytes;
    out->queued_jobs = e->queue.size();
  }
  return LC_OK;
}

lc_status lc_get_tuning(lc_engine* e, lc_tuning* out) {
  if (!e || !out) return fail(LC_ERR_INVALID_ARG, "null argument");
  const Tunables t = e->tuning();
  out->ctas_per_job = t.ctas_per_job;
  out->merge_items = t.merge_items;
  out->merge_threads = t.merge_threads;
  return LC_OK;
}

lc_status lc_set_tuning(lc_engine* e, const lc_tuning* t) {
  if (!e || !t) return fail(LC_ERR_INVALID_ARG, "null argument");
  if (t->merge_items < 1 || t->merge_items > 32 || t->merge_threads < 64 ||
      t->merge_threads > 1024 || t->merge_threads % 32 || t->ctas_per_job > 65535)
    return fail(LC_ERR_INVALID_ARG, "tuning out of range");
  std::lock_guard<std::mutex> g(e->tun_mu);
  e->tun.ctas_per_job = t->ctas_per_job;
  e->tun.merge_items = t->merge_items;
  e->tun.merge_threads = t->merge_threads;
  return LC_OK;
}

lc_status lc_autotune(lc_engine* e, int32_t n, const lc_job_desc* descs, int32_t repeats,
                      lc_tuning* chosen) {
  if (!e || n <= 0 || !descs || !chosen) return fail(LC_ERR_INVALID_ARG, "null argument");
  if (repeats < 1) repeats = 1;
  // outputs stay on the device: the tuner only needs the device time
  std::vector<lc_job_desc> d(descs, descs + n);
  for (auto& x : d) x.outputs_on_device = 1;
  std::vector<lc_job*> jobs(n, nullptr);
  // median device time of the whole set under one setting
  auto time_of = [&](const Tunables& t, double* ms) -> lc_status {
    {
      std::lock_guard<std::mutex> g(e->tun_mu);
      e->tun = t;
    }
    std::vector<double> v;
    for (int32_t r = 0; r < repeats + 1; r++) {  // the first run captures the graphs
      std::fill(jobs.begin(), jobs.end(), nullptr);
      lc_status s = lc_compact_batch(e, n, d.data(), jobs.data());
      double tot = 0;
      for (int32_t i = 0; i < n; i++) {
        if (jobs[i] && i % (int32_t)e->max_batch == 0) tot += jobs[i]->device_ms;  // per batch
        lc_job_release(jobs[i]);
      }
      if (s != LC_OK) return s;
      if (r > 0) v.push_back(tot);
    }
    std::sort(v.begin(), v.end());
    *ms = v[v.size() / 2];
    return LC_OK;
  };
  const Tunables saved = e->tuning();
  Tunables best = saved;
  double best_ms = 0;
  lc_status s = time_of(best, &best_ms);
  // coordinate search: merge tile (threads x items per thread), then CTAs per job
  const uint32_t threads[] = {128, 256, 512};
  const uint32_t items[] = {4, 8, 16};
  for (uint32_t th : threads)
    for (uint32_t it : items) {
      if (s != LC_OK) break;
      Tunables t = best;
      t.merge_threads = th;
      t.merge_items = it;
      if (t.merge_threads == best.merge_threads && t.merge_items == best.merge_items) continue;
      double ms;
      s = time_of(t, &ms);
      if (s == LC_OK && ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
  const uint32_t ctas[] = {0, 4, 16, 64, 256};
  for (uint32_t c : ctas) {
    if (s != LC_OK) break;
    if (c == best.ctas_per_job) continue;
    Tunables t = best;
    t.ctas_per_job = c;
    double ms;
    s = time_of(t, &ms);
    if (s == LC_OK && ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  std::lock_guard<std::mutex> g(e->tun_mu);
  e->tun = s == LC_OK ? best : saved;
  if (s != LC_OK) return s;
  chosen->ctas_per_job = best.ctas_per_job;
  chosen->merge_items = best.merge_items;
  chosen->merge_threads = best.merge_threads;
  return LC_OK;
}

lc_status lc_build_table(lc_engine* e, const lc_table_options* opt, int64_t n,
                         const uint8_t* keys, const uint64_t* key_offsets, const uint8_t* values,
                         const uint64_t* value_offsets, int32_t on_device, lc_job_out* out,
                         lc_job** job_out) {
  if (!e || !opt || !out || !job_out || n < 0 || !key_offsets || !value_offsets)
    return fail(LC_ERR_INVALID_ARG, "null argument");
  if (opt->block_size == 0 || opt->restart_interval == 0)
    return fail(LC_ERR_INVALID_ARG, "zero block size or restart interval");
  lc_job* j = new (std::nothrow) lc_job();
  if (!j) return fail(LC_ERR_NO_MEMORY, "job");
  j->eng = e;
  j->kind = 1;
  j->opt = *opt;
  j->bn = n;
  j->bkeys = keys;
  j->bvals = values;
  j->bkoffs = key_offsets;
  j->bvoffs = value_offsets;
  j->inputs_on_device = on_device;
  j->outputs_on_device = 0;
  lc_slot* slot = nullptr;
  try {
    CK(cudaSetDevice(e->device));
    slot = e->take_slot();
  } catch (const CudaError& ce) {
    delete j;
    return fail(LC_ERR_CUDA, std::string(ce.what) + ": " + cudaGetErrorString(ce.e));
  }
  run_build(j, *slot);
  e->put_slot(slot);
  j->done = true;
  if (j->status != LC_OK) {
    lc_status r = fail(j->status, j->err);
    lc_job_release(j);
    *job_out = nullptr;
    return r;
  }
  fill_out(j, out);
  *job_out = j;
  return LC_OK;
}

lc_status lc_crc32c(lc_engine* e, const uint8_t* data, uint64_t n, int32_t on_device,
                    uint32_t* masked_crc) {
  if (!e || !masked_crc || (n && !data)) return fail(LC_ERR_INVALID_ARG, "null argument");
  cudaStream_t st = nullptr;
  lc_slot* slot = nullptr;
  std::vector<void*> ptrs;
  try {
    CK(cudaSetDevice(e->device));
    slot = e->take_slot();
    st = slot->st;
    const uint8_t* d_data = data;
    const uint32_t chunks = crc32c_chunk_count(n);
    void* p = nullptr;
    if (!on_device && n) {
      CK(cudaMallocAsync(&p, n, st));
      ptrs.push_back(p);
      CK(cudaMemcpyAsync(p, data, n, cudaMemcpyHostToDevice, st));
      d_data = (const uint8_t*)p;
    }
    // scratch: one register per chunk, the ticket counter, the result
    CK(cudaMallocAsync(&p, ((size_t)chunks + 2) * sizeof(uint32_t), st));
    ptrs.push_back(p);
    uint32_t* partials = (uint32_t*)p;
    uint32_t* counter = partials + chunks;
    uint32_t* d_out = counter + 1;
    CK(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
    launch_crc32c_chunks(d_data, n, partials, counter, d_out, st);
    CK(cudaGetLastError());
    uint32_t h = 0;
    CK(cudaMemcpyAsync(&h, d_out, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    for (void* q : ptrs) CK(cudaFreeAsync(q, st));
    ptrs.clear();
    CK(cudaStreamSynchronize(st));
    e->put_slot(slot);
    *masked_crc = h;
    return LC_OK;
  } catch (const CudaError& ce) {
    if (slot) {
      for (void* q : ptrs) cudaFreeAsync(q, st);
      cudaStreamSynchronize(st);
      e->put_slot(slot);
    }
    return fail(LC_ERR_CUDA, std::string(ce.what) + ": " + cudaGetErrorString(ce.e));
  }
}

}  // extern "C"
