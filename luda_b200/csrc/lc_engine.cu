// Host orchestration and the C ABI (include/luda_b200.h).
//
// One job runs as a sequence of kernels on one CUDA stream:
//   upload -> table/index parse -> block count -> [sync: entry and key totals]
//   -> decode -> merge rounds -> drop rule + grandparent cuts -> survivors
//   -> entry sizes -> block chain -> blocks -> files -> layout
//   -> [sync: file count and output size] -> encode -> download -> [sync]
// Device memory comes from the device's stream-ordered pool (cudaMallocAsync),
// whose release threshold is raised so freed blocks are reused across jobs.
// Asynchronous jobs are served by worker threads, one stream each; a job is
// admitted only while the estimated device memory of the jobs in flight stays
// under the engine's budget.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
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

struct PinnedCache {
  std::mutex mu;
  std::vector<std::pair<uint8_t*, uint64_t>> free_list;
  uint8_t* take(uint64_t n, uint64_t* cap) {
    {
      std::lock_guard<std::mutex> g(mu);
      size_t best = free_list.size();
      for (size_t i = 0; i < free_list.size(); i++)
        if (free_list[i].second >= n &&
            (best == free_list.size() || free_list[i].second < free_list[best].second))
          best = i;
      if (best != free_list.size()) {
        auto r = free_list[best];
        free_list.erase(free_list.begin() + best);
        *cap = r.second;
        return r.first;
      }
    }
    uint64_t c = std::max<uint64_t>(n, 1 << 20);
    c = (c + (1 << 20) - 1) & ~uint64_t((1 << 20) - 1);
    void* p = nullptr;
    if (cudaMallocHost(&p, c) != cudaSuccess) return nullptr;
    *cap = c;
    return (uint8_t*)p;
  }
  void give(uint8_t* p, uint64_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> g(mu);
    free_list.emplace_back(p, cap);
  }
  void clear() {
    std::lock_guard<std::mutex> g(mu);
    for (auto& f : free_list) cudaFreeHost(f.first);
    free_list.clear();
  }
};

}  // namespace

struct lc_engine {
  int device = 0;
  uint64_t budget = 40ull << 30;
  int max_inflight = 4;
  uint32_t flags = 0;
  uint32_t* crc_xpow = nullptr;
  PinnedCache pinned;
  std::mutex mu;
  std::condition_variable cv;
  std::condition_variable admit_cv;
  std::deque<lc_job*> queue;
  std::vector<std::thread> workers;
  bool stop = false;
  uint64_t inflight_bytes = 0;
  std::mutex stream_mu;
  std::vector<cudaStream_t> free_streams;
  cudaStream_t get_stream() {
    {
      std::lock_guard<std::mutex> g(stream_mu);
      if (!free_streams.empty()) {
        cudaStream_t s = free_streams.back();
        free_streams.pop_back();
        return s;
      }
    }
    cudaStream_t s;
    cudaSetDevice(device);
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    return s;
  }
  void put_stream(cudaStream_t s) {
    std::lock_guard<std::mutex> g(stream_mu);
    free_streams.push_back(s);
  }
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
  // build-table inputs
  int64_t bn = 0;
  const uint8_t *bkeys = nullptr, *bvals = nullptr;
  const uint64_t *bkoffs = nullptr, *bvoffs = nullptr;
  // results
  lc_status status = LC_OK;
  std::string err;
  uint8_t* h_out = nullptr;
  uint64_t h_out_cap = 0;
  uint8_t* d_out = nullptr;  // kept when outputs_on_device
  std::vector<uint64_t> file_offset, file_size, file_entries, small_off, large_off;
  std::vector<uint32_t> small_len, large_len;
  std::vector<uint8_t> key_bytes;
  uint64_t bytes_in = 0, bytes_out = 0, entries_in = 0, entries_out = 0;
  double device_ms = 0;
  uint32_t launches = 0;
  std::vector<float> phase_ms;
  uint64_t key_bytes_in = 0, kept_key_bytes = 0, kept_value_bytes = 0;
  uint64_t est_bytes = 0;
  // completion
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
};

namespace {

// Device allocations of one job: a bump allocator over a few large chunks of
// the stream-ordered pool (one cudaMallocAsync per 64 MiB instead of one per
// array), all freed in stream order at the end.  Sub-allocations are
// 256-byte aligned and padded so that 16-byte vector loads may run past the
// end of an array.
struct DevAlloc {
  static constexpr uint64_t kChunkBytes = 64ull << 20;
  cudaStream_t st;
  std::vector<void*> ptrs;
  uint8_t* cur = nullptr;
  uint64_t left = 0;
  explicit DevAlloc(cudaStream_t s) : st(s) {}
  template <typename T>
  T* get(uint64_t n) {
    const uint64_t bytes = (std::max<uint64_t>(n, 1) * sizeof(T) + 16 + 255) & ~uint64_t(255);
    if (bytes > left) {
      const uint64_t c = std::max(bytes, kChunkBytes);
      void* p = nullptr;
      CK(cudaMallocAsync(&p, c, st));
      ptrs.push_back(p);
      cur = (uint8_t*)p;
      left = c;
    }
    T* r = (T*)cur;
    cur += bytes;
    left -= bytes;
    return r;
  }
  // a separate allocation (e.g. an output that outlives the job)
  uint8_t* own(uint64_t bytes) {
    void* p = nullptr;
    CK(cudaMallocAsync(&p, std::max<uint64_t>(bytes, 16) + 64, st));
    ptrs.push_back(p);
    return (uint8_t*)p;
  }
  void release(void* keep = nullptr) {
    for (void* p : ptrs)
      if (p != keep) cudaFreeAsync(p, st);
    ptrs.clear();
    cur = nullptr;
    left = 0;
  }
};

void check_launch() { CK(cudaGetLastError()); }

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
  cudaStream_t st = nullptr;
  std::vector<std::pair<int, cudaEvent_t>> evs;  // (phase ended here, or -1), in order
  PhaseTimer(bool enable, cudaStream_t s) : on(enable), st(s) {}
  ~PhaseTimer() {
    for (auto& e : evs) cudaEventDestroy(e.second);
  }
  void record(int tag) {
    if (!on) return;
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, st));
    evs.emplace_back(tag, e);
  }
  // a phase runs from the previous recorded event to its mark
  void start() { record(-1); }
  void mark(int p) { record(p); }
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
    case kErrLimit: return "engine limit exceeded";
    default: return "unknown";
  }
}

void check_counters(const Counters& c) {
  if (c.error) {
    lc_status s = (c.error == kErrLimit || c.error == kErrArenaOverflow) ? LC_ERR_UNSUPPORTED
                                                                         : LC_ERR_CORRUPT;
    throw StatusError{s, std::string(err_name(c.error)) + " (detail " +
                             std::to_string(c.error_detail) + ")"};
  }
}

void read_counters(Counters* h, const Counters* d, cudaStream_t st) {
  CK(cudaMemcpyAsync(h, d, sizeof(Counters), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  check_counters(*h);
}

uint32_t bloom_k(int bpk) {
  // util/bloom.cc:20-24
  size_t k = static_cast<size_t>(bpk * 0.69);
  if (k < 1) k = 1;
  if (k > 30) k = 30;
  return (uint32_t)k;
}

// Survivors (k_ids, counters n_kept / n_triggers set) -> encoded files.
void encode_tail(lc_job* j, JobDev& J, DevAlloc& A, uint64_t N, Counters* hc, cudaStream_t st,
                 PhaseTimer& T, uint32_t max_klen) {
  J.k_a = A.get<uint32_t>(N);
  J.k_b = A.get<uint32_t>(N);
  J.k_shared = A.get<uint32_t>(N);
  J.k_next = A.get<uint32_t>(N);
  J.k_bstart = A.get<uint8_t>(N + 1);
  J.k_block = A.get<uint32_t>(N + 1);
  CK(cudaMemsetAsync(J.k_bstart, 0, N + 1, st));
  J.chunk = kChunk;
  J.chain_smem_words = 12 * 1024;  // 48 KiB
  const uint64_t chunks = (N + kChunk - 1) / kChunk + 1;
  J.chunk_table = A.get<uint32_t>(chunks * kChunk);
  J.chunk_entry = A.get<uint32_t>(chunks);
  uint64_t* scratch64 = A.get<uint64_t>(scan_scratch_elems(N + 1));
  uint32_t* scratch32 = A.get<uint32_t>(scan_scratch_elems(N + 1));

  launch_sizes(J, N, st);
  launch_next(J, N, st);
  launch_chain(J, N, st);
  scan_exclusive<uint8_t, uint32_t>(J.k_bstart, J.k_block, &J.ctr->n_kept, N, scratch32,
                                    &J.ctr->n_blocks_out, st);
  J.b_first = A.get<uint32_t>(N + 1);
  launch_block_list(J, N, st);
  J.b_size = A.get<uint32_t>(N);
  uint32_t* tmp32 = A.get<uint32_t>(N);
  J.b_cum = A.get<uint64_t>(N + 1);
  launch_block_sizes(J, tmp32, N, st);
  scan_exclusive<uint32_t, uint64_t>(tmp32, J.b_cum, &J.ctr->n_blocks_out, N, scratch64,
                                     nullptr, st);
  J.cap_files = (uint32_t)std::min<uint64_t>(N + 1, 64 + J.cap_triggers +
                                                         (8 * (J.in_size + J.cap_key_bytes) + N * 64) /
                                                             std::max<uint64_t>(1, J.max_file_size));
  J.files = A.get<FileOut>(J.cap_files);
  J.b_fnext = A.get<uint32_t>(N);
  J.t_blocks = A.get<uint32_t>(J.cap_triggers);
  launch_files(J, N, st);
  J.b_file = A.get<uint32_t>(N);
  J.b_off = A.get<uint64_t>(N);
  J.b_isize = A.get<uint32_t>(N);
  J.b_icum = A.get<uint64_t>(N + 1);
  J.b_sep = A.get<uint32_t>(N);
  J.b_ilen = A.get<uint32_t>(N);
  J.b_gbytes = A.get<uint32_t>(N);
  J.b_gcum = A.get<uint64_t>(N + 1);
  J.b_gkeys = A.get<uint32_t>(N);
  launch_block_layout(J, N, st);
  scan_exclusive<uint32_t, uint64_t>(J.b_gbytes, J.b_gcum, &J.ctr->n_blocks_out, N, scratch64,
                                     nullptr, st);
  scan_exclusive<uint32_t, uint64_t>(J.b_isize, J.b_icum, &J.ctr->n_blocks_out, N, scratch64,
                                     nullptr, st);
  // Output capacity, bounded without waiting for the layout: every survivor
  // costs at most its key, its value and 15 header bytes; every block at most
  // 4 bytes of restart word per entry, 9 bytes of count and trailer, one index
  // entry (key + 31) and a filter share; every file 256 bytes of metaindex,
  // footer and trailers.  The layout kernel checks the real size against it.
  const uint64_t bpk = j->opt.bits_per_key > 0 ? (uint64_t)j->opt.bits_per_key : 0;
  J.cap_out = J.in_size + 2 * J.cap_key_bytes + N * (80 + max_klen + (bpk + 7) / 8) +
              (uint64_t)J.cap_files * 256 + (J.in_size + J.cap_key_bytes) / 256 + 65536;
  J.out = A.own(J.cap_out);
  launch_file_layout(J, st);
  check_launch();
  T.mark(kPartition);
  launch_encode_blocks(J, N, st);
  T.mark(kEncodeBlocks);
  launch_encode_rest(J, N, J.cap_files, st);
  T.mark(kEncodeMeta);
  // smallest / largest key of every file, gathered on the device
  const uint64_t key_cap = 2ull * J.cap_files * max_klen;
  uint8_t* d_keys = A.get<uint8_t>(key_cap + 1);
  uint64_t* d_koff = A.get<uint64_t>(2ull * J.cap_files + 1);
  launch_file_keys(J, J.cap_files, d_keys, d_koff, st);
  check_launch();
  std::vector<FileOut> files(J.cap_files);
  std::vector<uint64_t> koff(2ull * J.cap_files + 1);
  j->key_bytes.resize(key_cap + 1);
  CK(cudaMemcpyAsync(hc, J.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(files.data(), J.files, J.cap_files * sizeof(FileOut), cudaMemcpyDeviceToHost,
                     st));
  CK(cudaMemcpyAsync(koff.data(), d_koff, koff.size() * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(j->key_bytes.data(), d_keys, key_cap + 1, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  check_counters(*hc);
  const uint32_t nf = hc->n_files;
  const uint64_t nbytes = hc->bytes_out;
  if (!j->outputs_on_device && nbytes) {
    j->h_out = j->eng->pinned.take(nbytes, &j->h_out_cap);
    if (!j->h_out) throw StatusError{LC_ERR_NO_MEMORY, "pinned host buffer"};
    CK(cudaMemcpyAsync(j->h_out, J.out, nbytes, cudaMemcpyDeviceToHost, st));
  }
  j->file_offset.resize(nf);
  j->file_size.resize(nf);
  j->file_entries.resize(nf);
  j->small_off.resize(nf);
  j->large_off.resize(nf);
  j->small_len.resize(nf);
  j->large_len.resize(nf);
  for (uint32_t f = 0; f < nf; f++) {
    j->file_offset[f] = files[f].out_off;
    j->file_size[f] = files[f].size;
    j->file_entries[f] = files[f].end_kept - files[f].first_kept;
    j->small_off[f] = koff[2 * f];
    j->small_len[f] = (uint32_t)(koff[2 * f + 1] - koff[2 * f]);
    j->large_off[f] = koff[2 * f + 1];
    j->large_len[f] = (uint32_t)(koff[2 * f + 2] - koff[2 * f + 1]);
  }
  T.mark(kDownload);
  j->bytes_out = nbytes;
  j->entries_out = hc->n_kept;
  j->kept_key_bytes = hc->kept_key_bytes;
  j->kept_value_bytes = hc->kept_value_bytes;
  if (j->outputs_on_device) j->d_out = J.out;
}

void fill_common(JobDev& J, const lc_job* j, lc_engine* e) {
  memset(&J, 0, sizeof(J));
  J.block_size = j->opt.block_size;
  J.restart_interval = j->opt.restart_interval;
  J.bits_per_key = j->opt.bits_per_key;
  J.bloom_k = j->opt.bits_per_key > 0 ? bloom_k(j->opt.bits_per_key) : 0;
  J.max_file_size = j->opt.max_file_size;
  J.smallest_snapshot = j->smallest_snapshot;
  J.max_gp_overlap = (int64_t)(10 * j->opt.max_file_size);  // db/version_set.cc:31-33
  J.crc_xpow = e->crc_xpow;
  J.crc_xpow_n = kCrcXpowN;
}

void run_compaction(lc_job* j, cudaStream_t st) {
  lc_engine* e = j->eng;
  DevAlloc A(st);
  PhaseTimer T((e->flags & LC_FLAG_PHASE_TIMING) != 0, st);
  const uint32_t launches0 = launches_on_this_thread();
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  try {
    CK(cudaEventRecord(ev0, st));
    T.start();
    JobDev J;
    fill_common(J, j, e);
    const uint32_t nt = (uint32_t)j->tables.size();
    std::vector<TableDesc> td(nt);
    uint32_t run = 0, in_run = 0;
    for (uint32_t t = 0; t < nt; t++) {
      while (run < j->run_counts.size() && in_run >= (uint32_t)j->run_counts[run]) {
        run++;
        in_run = 0;
      }
      td[t].run = run;
      td[t].size = j->tables[t].size;
      in_run++;
    }
    J.n_tables = nt;
    J.n_runs = (uint32_t)j->run_counts.size();
    // input placement
    uint8_t* d_in = nullptr;
    uint64_t in_size = 0;
    bool zero_copy = false;
    if (j->inputs_on_device) {
      uintptr_t lo = ~uintptr_t(0), hi = 0;
      for (auto& t : j->tables) {
        lo = std::min(lo, (uintptr_t)t.data);
        hi = std::max(hi, (uintptr_t)t.data + (uintptr_t)t.size);
      }
      if (nt && hi - lo < (1ull << 32)) {
        zero_copy = true;
        d_in = (uint8_t*)lo;
        in_size = hi - lo;
        for (uint32_t t = 0; t < nt; t++) td[t].off = (uintptr_t)j->tables[t].data - lo;
      }
    }
    if (!zero_copy) {
      for (uint32_t t = 0; t < nt; t++) {
        td[t].off = in_size;
        in_size += round16(td[t].size);
      }
      if (in_size >= (1ull << 32))
        throw StatusError{LC_ERR_UNSUPPORTED, "input of one job must be below 4 GiB"};
      d_in = A.get<uint8_t>(in_size + 16);
      for (uint32_t t = 0; t < nt; t++) {
        if (!j->tables[t].size) continue;
        CK(cudaMemcpyAsync(d_in + td[t].off, j->tables[t].data, j->tables[t].size,
                           j->inputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           st));
      }
    }
    J.in = d_in;
    J.in_size = in_size;
    J.in_end = d_in + in_size + (zero_copy ? 0 : 16);
    TableDesc* d_td = A.get<TableDesc>(nt);
    CK(cudaMemcpyAsync(d_td, td.data(), nt * sizeof(TableDesc), cudaMemcpyHostToDevice, st));
    J.tables = d_td;
    // grandparents
    J.n_gp = (uint32_t)j->gp_largest.size();
    {
      std::vector<uint64_t> off(J.n_gp + 1, 0), pre(J.n_gp + 1, 0);
      std::string kb;
      for (uint32_t g = 0; g < J.n_gp; g++) {
        kb += j->gp_largest[g];
        off[g + 1] = kb.size();
        pre[g + 1] = pre[g] + j->gp_size[g];
      }
      uint8_t* dk = A.get<uint8_t>(kb.size() + 1);
      uint64_t* doff = A.get<uint64_t>(off.size());
      uint64_t* dpre = A.get<uint64_t>(pre.size());
      if (!kb.empty()) CK(cudaMemcpyAsync(dk, kb.data(), kb.size(), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(doff, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(dpre, pre.data(), pre.size() * 8, cudaMemcpyHostToDevice, st));
      J.gp_keys = dk;
      J.gp_key_off = doff;
      J.gp_prefix = dpre;
    }
    // base-level files, grouped by level (given in level then key order)
    {
      const uint32_t nb = (uint32_t)j->base_level.size();
      std::vector<uint32_t> lvl_begin;
      std::vector<uint64_t> so(nb), lo_(nb);
      std::vector<uint32_t> sl(nb), ll(nb);
      std::string kb;
      for (uint32_t i = 0; i < nb; i++) {
        if (i == 0 || j->base_level[i] != j->base_level[i - 1]) lvl_begin.push_back(i);
        so[i] = kb.size();
        sl[i] = (uint32_t)j->base_small[i].size();
        kb += j->base_small[i];
        lo_[i] = kb.size();
        ll[i] = (uint32_t)j->base_large[i].size();
        kb += j->base_large[i];
      }
      lvl_begin.push_back(nb);
      J.n_base_levels = nb ? (uint32_t)lvl_begin.size() - 1 : 0;
      uint32_t* d_lb = A.get<uint32_t>(lvl_begin.size());
      uint8_t* d_kb = A.get<uint8_t>(kb.size() + 1);
      uint64_t* d_so = A.get<uint64_t>(nb + 1);
      uint64_t* d_lo = A.get<uint64_t>(nb + 1);
      uint32_t* d_sl = A.get<uint32_t>(nb + 1);
      uint32_t* d_ll = A.get<uint32_t>(nb + 1);
      CK(cudaMemcpyAsync(d_lb, lvl_begin.data(), lvl_begin.size() * 4, cudaMemcpyHostToDevice, st));
      if (nb) {
        CK(cudaMemcpyAsync(d_kb, kb.data(), kb.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_so, so.data(), nb * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_lo, lo_.data(), nb * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_sl, sl.data(), nb * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_ll, ll.data(), nb * 4, cudaMemcpyHostToDevice, st));
      }
      J.base_level_begin = d_lb;
      J.base_keys = d_kb;
      J.base_small_off = d_so;
      J.base_large_off = d_lo;
      J.base_small_len = d_sl;
      J.base_large_len = d_ll;
    }
    J.ctr = A.get<Counters>(1);
    CK(cudaMemsetAsync(J.ctr, 0, sizeof(Counters), st));

    // blocks of the input tables (capacity: a data block with its trailer and
    // index entry takes at least 13 bytes)
    uint64_t cap_blk = 1;
    for (auto& t : td) cap_blk += t.size / 13 + 1;
    J.cap_blocks_in = cap_blk;
    J.tbl_nblocks = A.get<uint32_t>(nt);
    J.tbl_block_base = A.get<uint64_t>(nt + 1);
    J.blk_off = A.get<uint64_t>(cap_blk);
    J.blk_size = A.get<uint32_t>(cap_blk);
    J.blk_run = A.get<uint32_t>(cap_blk);
    J.blk_nent = A.get<uint32_t>(cap_blk);
    J.blk_ent_base = A.get<uint64_t>(cap_blk + 1);
    J.blk_kbytes = A.get<uint64_t>(cap_blk);
    J.blk_key_base = A.get<uint64_t>(cap_blk + 1);
    uint64_t* scratch = A.get<uint64_t>(scan_scratch_elems(cap_blk + nt + 1));
    J.run_entry_begin_w = A.get<uint64_t>(J.n_runs + 1);
    J.run_entry_begin = J.run_entry_begin_w;

    T.mark(kUpload);
    Counters hc;
    if (nt) {
      launch_table_index_count(J, st);
      scan_exclusive<uint32_t, uint64_t>(J.tbl_nblocks, J.tbl_block_base, nullptr, nt, scratch,
                                         &J.ctr->n_blocks_in, st);
      launch_table_index_entries(J, st);
      launch_block_count(J, cap_blk, st);
      scan_exclusive<uint32_t, uint64_t>(J.blk_nent, J.blk_ent_base, &J.ctr->n_blocks_in, cap_blk,
                                         scratch, &J.ctr->n_entries_in, st);
      scan_exclusive<uint64_t, uint64_t>(J.blk_kbytes, J.blk_key_base, &J.ctr->n_blocks_in,
                                         cap_blk, scratch, &J.ctr->key_bytes_in, st);
    }
    launch_run_bounds(J, st);
    check_launch();
    T.mark(kParse);
    read_counters(&hc, J.ctr, st);
    if (hc.n_blocks_in > cap_blk) throw StatusError{LC_ERR_CORRUPT, "more blocks than bytes allow"};
    const uint64_t N = hc.n_entries_in, K = hc.key_bytes_in;
    if (N >= (1ull << 32) - 2 || K >= (1ull << 32))
      throw StatusError{LC_ERR_UNSUPPORTED, "more than 2^32 entries or key bytes in one job"};
    j->entries_in = N;
    j->key_bytes_in = K;

    J.keys = A.get<uint8_t>(K + 16);
    J.cap_key_bytes = K;
    J.cap_entries = N;
    J.e_koff = A.get<uint32_t>(N);
    J.e_klen = A.get<uint32_t>(N);
    J.e_voff = A.get<uint32_t>(N);
    J.e_vlen = A.get<uint32_t>(N);
    J.e_pfx = A.get<uint64_t>(N);
    T.start();
    launch_block_decode(J, hc.n_blocks_in, st);
    T.mark(kDecode);

    // merge rounds
    J.m_ids = A.get<uint32_t>(N);
    J.m_tmp = A.get<uint32_t>(N);
    launch_iota(J.m_ids, N, st);
    uint32_t* src = J.m_ids;
    uint32_t* dst = J.m_tmp;
    for (uint32_t w = 1; w < J.n_runs; w *= 2) {
      launch_merge_round(J, src, dst, w, N, st);
      std::swap(src, dst);
    }
    J.m_ids = src;
    J.m_tmp = dst;
    T.mark(kMerge);

    // drop rule, grandparent cuts, survivors
    J.keep = A.get<uint8_t>(N);
    J.gp_idx = A.get<uint32_t>(J.n_gp ? N : 1);
    J.kept_pos = A.get<uint32_t>(N + 1);
    J.cap_triggers = J.n_gp + 1;
    J.triggers = A.get<uint32_t>(J.cap_triggers);
    J.k_ids = A.get<uint32_t>(N);
    J.k_forced = A.get<uint8_t>(N + 1);
    uint32_t* scratch32 = A.get<uint32_t>(scan_scratch_elems(N + 1));
    launch_drop(J, N, st);
    launch_triggers(J, N, A.get<uint32_t>(J.n_gp + 1), st);
    scan_exclusive<uint8_t, uint32_t>(J.keep, J.kept_pos, &J.ctr->n_entries_in, N, scratch32,
                                      &J.ctr->n_kept, st);
    launch_kept_compact(J, N, st);
    check_launch();
    T.mark(kDrop);
    encode_tail(j, J, A, N, &hc, st, T, std::max<uint32_t>(hc.max_klen, 8));
    CK(cudaEventRecord(ev1, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    j->device_ms = ms;
    T.collect(j->phase_ms);
    j->launches = launches_on_this_thread() - launches0;
    A.release(j->d_out);
    CK(cudaStreamSynchronize(st));
  } catch (...) {
    cudaStreamSynchronize(st);
    A.release();
    j->d_out = nullptr;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    throw;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
}

void run_build(lc_job* j, cudaStream_t st) {
  lc_engine* e = j->eng;
  DevAlloc A(st);
  PhaseTimer T((e->flags & LC_FLAG_PHASE_TIMING) != 0, st);
  const uint32_t launches0 = launches_on_this_thread();
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  try {
    CK(cudaEventRecord(ev0, st));
    T.start();
    JobDev J;
    fill_common(J, j, e);
    J.max_file_size = ~0ull;  // BuildTable writes one file
    J.max_gp_overlap = 0;
    const uint64_t N = (uint64_t)j->bn;
    uint64_t kb, vb;
    if (j->inputs_on_device) {
      CK(cudaMemcpyAsync(&kb, j->bkoffs + N, 8, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&vb, j->bvoffs + N, 8, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    } else {
      kb = j->bkoffs[N];
      vb = j->bvoffs[N];
    }
    if (kb >= (1ull << 32) || vb >= (1ull << 32) || N >= (1ull << 32) - 2)
      throw StatusError{LC_ERR_UNSUPPORTED, "table input beyond 4 GiB"};
    const cudaMemcpyKind kind = j->inputs_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    J.keys = A.get<uint8_t>(kb + 16);
    uint8_t* d_vals = A.get<uint8_t>(vb + 16);
    uint64_t* d_ko = A.get<uint64_t>(N + 1);
    uint64_t* d_vo = A.get<uint64_t>(N + 1);
    if (kb) CK(cudaMemcpyAsync(J.keys, j->bkeys, kb, kind, st));
    if (vb) CK(cudaMemcpyAsync(d_vals, j->bvals, vb, kind, st));
    CK(cudaMemcpyAsync(d_ko, j->bkoffs, (N + 1) * 8, kind, st));
    CK(cudaMemcpyAsync(d_vo, j->bvoffs, (N + 1) * 8, kind, st));
    J.in = d_vals;
    J.in_size = vb;
    J.in_end = d_vals + vb + 16;
    J.cap_key_bytes = kb;
    J.cap_entries = N;
    J.ctr = A.get<Counters>(1);
    CK(cudaMemsetAsync(J.ctr, 0, sizeof(Counters), st));
    Counters init{};
    init.n_kept = N;
    init.n_entries_in = N;
    CK(cudaMemcpyAsync(J.ctr, &init, sizeof(Counters), cudaMemcpyHostToDevice, st));
    J.e_koff = A.get<uint32_t>(N);
    J.e_klen = A.get<uint32_t>(N);
    J.e_voff = A.get<uint32_t>(N);
    J.e_vlen = A.get<uint32_t>(N);
    J.e_pfx = A.get<uint64_t>(N);
    J.k_ids = A.get<uint32_t>(N);
    J.k_forced = A.get<uint8_t>(N + 1);
    CK(cudaMemsetAsync(J.k_forced, 0, N + 1, st));
    J.cap_triggers = 1;
    J.triggers = A.get<uint32_t>(1);
    J.kept_pos = A.get<uint32_t>(N + 1);
    T.mark(kUpload);
    launch_entries_from_offsets(J, d_ko, d_vo, N, st);
    check_launch();
    T.mark(kDrop);
    Counters hc;
    j->entries_in = N;
    j->key_bytes_in = kb;
    uint32_t max_klen = 8;
    {
      std::vector<uint64_t> hk;
      const uint64_t* ko = j->bkoffs;
      if (j->inputs_on_device) {
        hk.resize(N + 1);
        CK(cudaMemcpyAsync(hk.data(), j->bkoffs, (N + 1) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ko = hk.data();
      }
      for (uint64_t i = 0; i < N; i++)
        max_klen = std::max<uint32_t>(max_klen, (uint32_t)(ko[i + 1] - ko[i]));
    }
    encode_tail(j, J, A, N, &hc, st, T, max_klen);
    CK(cudaEventRecord(ev1, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    j->device_ms = ms;
    T.collect(j->phase_ms);
    j->launches = launches_on_this_thread() - launches0;
    A.release(j->d_out);
    CK(cudaStreamSynchronize(st));
  } catch (...) {
    cudaStreamSynchronize(st);
    A.release();
    j->d_out = nullptr;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    throw;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
}

void execute(lc_job* j, cudaStream_t st) {
  try {
    CK(cudaSetDevice(j->eng->device));
    if (j->kind == 0) run_compaction(j, st);
    else run_build(j, st);
    j->status = LC_OK;
  } catch (const CudaError& ce) {
    j->status = LC_ERR_CUDA;
    j->err = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
  } catch (const StatusError& se) {
    j->status = se.s;
    j->err = se.msg;
  } catch (const std::bad_alloc&) {
    j->status = LC_ERR_NO_MEMORY;
    j->err = "host allocation failed";
  }
}

uint64_t estimate_bytes(const lc_job* j) {
  uint64_t in = 0;
  for (auto& t : j->tables) in += t.size;
  if (j->kind == 1) in = j->bkoffs && !j->inputs_on_device ? j->bkoffs[j->bn] + j->bvoffs[j->bn] : 0;
  return 24 * in + (64ull << 20);
}

void finish(lc_job* j) {
  std::lock_guard<std::mutex> g(j->mu);
  j->done = true;
  j->cv.notify_all();
}

void worker_main(lc_engine* e) {
  cudaSetDevice(e->device);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  while (true) {
    lc_job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv.wait(lk, [&] { return e->stop || !e->queue.empty(); });
      if (e->stop && e->queue.empty()) break;
      // admission against the device budget (head of line first)
      lc_job* head = e->queue.front();
      e->admit_cv.wait(lk, [&] {
        return e->stop || e->inflight_bytes == 0 || e->inflight_bytes + head->est_bytes <= e->budget;
      });
      if (e->queue.empty() || e->queue.front() != head) continue;
      e->queue.pop_front();
      j = head;
      e->inflight_bytes += j->est_bytes;
    }
    if (e->stop) {
      j->status = LC_ERR_SHUTDOWN;
    } else {
      execute(j, st);
    }
    {
      std::lock_guard<std::mutex> g(e->mu);
      e->inflight_bytes -= j->est_bytes;
    }
    e->admit_cv.notify_all();
    e->cv.notify_all();
    finish(j);
  }
  cudaStreamDestroy(st);
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
  j->outputs_on_device = d->outputs_on_device;
  for (auto& t : j->tables) j->bytes_in += t.size;
  return LC_OK;
}

void fill_out(lc_job* j, lc_job_out* o) {
  memset(o, 0, sizeof(*o));
  o->n_files = (int32_t)j->file_size.size();
  o->data = j->outputs_on_device ? j->d_out : j->h_out;
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
}

void host_crc_xpow(std::vector<uint32_t>& t) {
  t.resize(kCrcXpowN);
  uint32_t c = 0x80000000u;  // x^0
  for (uint32_t m = 0; m < kCrcXpowN; m++) {
    t[m] = c;
    for (int b = 0; b < 8; b++) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
  }
}

}  // namespace

extern "C" {

const char* lc_version(void) { return kVersion; }
const char* lc_last_error(void) { return g_last_error.c_str(); }

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
  if (cfg) {
    e->device = cfg->device;
    if (cfg->device_budget_bytes) e->budget = cfg->device_budget_bytes;
    if (cfg->max_inflight_jobs > 0) e->max_inflight = cfg->max_inflight_jobs;
    e->flags = cfg->flags;
  }
  try {
    CK(cudaSetDevice(e->device));
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, e->device));
    uint64_t thr = ~0ull;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    std::vector<uint32_t> t;
    host_crc_xpow(t);
    CK(cudaMalloc(&e->crc_xpow, t.size() * 4));
    CK(cudaMemcpy(e->crc_xpow, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
  } catch (const CudaError& ce) {
    std::string m = std::string(ce.what) + ": " + cudaGetErrorString(ce.e);
    delete e;
    return fail(LC_ERR_CUDA, m);
  }
  for (int i = 0; i < e->max_inflight; i++) e->workers.emplace_back(worker_main, e);
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
  for (auto s : e->free_streams) cudaStreamDestroy(s);
  e->pinned.clear();
  cudaFree(e->crc_xpow);
  delete e;
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
    e->queue.push_back(j);
  }
  e->cv.notify_one();
  *out = j;
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
  if (j->d_out) {
    // the job has completed; return the output to the stream-ordered pool
    cudaSetDevice(j->eng->device);
    cudaFreeAsync(j->d_out, 0);
  }
  delete j;
}

lc_status lc_compact(lc_engine* e, const lc_job_desc* desc, lc_job_out* out, lc_job** job_out) {
  if (!e || !desc || !out || !job_out) return fail(LC_ERR_INVALID_ARG, "null argument");
  lc_job* j = new (std::nothrow) lc_job();
  if (!j) return fail(LC_ERR_NO_MEMORY, "job");
  j->eng = e;
  lc_status s = copy_desc(j, desc);
  if (s != LC_OK) {
    delete j;
    return s;
  }
  cudaSetDevice(e->device);
  cudaStream_t st = e->get_stream();
  execute(j, st);
  e->put_stream(st);
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
  cudaSetDevice(e->device);
  cudaStream_t st = e->get_stream();
  execute(j, st);
  e->put_stream(st);
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
  std::vector<void*> ptrs;
  try {
    CK(cudaSetDevice(e->device));
    st = e->get_stream();
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
    e->put_stream(st);
    *masked_crc = h;
    return LC_OK;
  } catch (const CudaError& ce) {
    if (st) {
      for (void* q : ptrs) cudaFreeAsync(q, st);
      cudaStreamSynchronize(st);
      e->put_stream(st);
    }
    return fail(LC_ERR_CUDA, std::string(ce.what) + ": " + cudaGetErrorString(ce.e));
  }
}

}  // extern "C"
