// DBImpl::DoCompactionWork served by the luda_b200 engine (include/luda_b200.h).
//
// This is the host side a LevelDB (LUDA) maintainer adds: the body below
// replaces the reference's CPU definition (db/db_impl.cc:1060-1224) and LUDA's
// GPU definition (db/db_impl.cc:1229-1591).  It is compiled inside
// db/db_impl.cc's own translation unit, at the place of the CPU definition
// (CompactionState, db/db_impl.cc:195-227, is private to that file), with
// include/luda_b200.h included ahead of the file.  The compaction loop itself
// -- merge, drop rule, output split, table encoding -- runs as one lc_job on
// the GPU; everything around it stays as the reference has it:
//
//   * the smallest snapshot, the unlocked work and the re-lock before install
//     (db/db_impl.cc:1073-1080, 1211-1212);
//   * memtable compaction while the work runs, ahead of everything else
//     ("Prioritize immutable compaction work", :1090-1102): here between
//     short waits on the GPU job instead of between input entries;
//   * the shutdown check (:1090, :1189-1190): a job already on the GPU runs to
//     its end, its outputs are dropped and the status is the reference's;
//   * output files numbered under mutex_ and protected in pending_outputs_
//     (OpenCompactionOutputFile, :966-989), written, synced, closed and read
//     back through the table cache (FinishCompactionOutputFile, :991-1038);
//   * CompactionStats (:1199-1211), InstallCompactionResults (:1040-1056) and
//     RecordBackgroundError (:915-921).
//
// The engine is created on first use, one per process, on the CUDA device
// named by LUDA_B200_DEVICE (default 0).  Options the engine cannot reproduce
// byte for byte (a comparator other than the bytewise one, a filter policy
// other than the built-in bloom filter) fail the compaction with
// Status::NotSupported: there is no CPU fallback.

namespace luda_b200_host {

// One engine per process, created on first use.
inline lc_engine* Engine(Status* s) {
  static std::mutex mu;
  static lc_engine* engine = nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (engine == nullptr) {
    lc_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    const char* dev = getenv("LUDA_B200_DEVICE");
    cfg.device = dev ? atoi(dev) : 0;
    cfg.max_inflight_jobs = 1;
    const lc_status st = lc_engine_create(&cfg, &engine);
    if (st != LC_OK) {
      *s = Status::IOError("luda_b200 engine", lc_last_error());
      engine = nullptr;
    }
  }
  return engine;
}

// Compactions the engine has served in this process (for tests).
inline std::atomic<uint64_t>& ServedCount() {
  static std::atomic<uint64_t> n{0};
  return n;
}

inline Status ToStatus(lc_status st) {
  if (st == LC_OK) return Status::OK();
  const char* msg = lc_last_error();
  switch (st) {
    case LC_ERR_CORRUPT: return Status::Corruption("luda_b200", msg);
    case LC_ERR_INVALID_ARG: return Status::InvalidArgument("luda_b200", msg);
    case LC_ERR_UNSUPPORTED: return Status::NotSupported("luda_b200", msg);
    default: return Status::IOError("luda_b200", msg);
  }
}

// bits_per_key of the built-in bloom policy, read back from the filter it
// makes for 64 keys: max(64, 64 * bits_per_key) bits plus the probe-count
// byte (util/bloom.cc:28-54).  `policy` is the sanitized options' policy,
// which takes internal keys and hands their user keys to the user's policy
// (db/dbformat.cc:105-115).  0 for no policy; -1 for any other policy.
inline int BloomBitsPerKey(const FilterPolicy* policy) {
  if (policy == nullptr) return 0;
  if (strcmp(policy->Name(), "leveldb.BuiltinBloomFilter2") != 0) return -1;
  std::vector<std::string> keys(64);
  std::vector<Slice> slices(64);
  for (int i = 0; i < 64; i++) {
    keys[i] = "k" + std::to_string(i) + std::string(8, '\0');  // user key + tag
    slices[i] = keys[i];
  }
  std::string dst;
  policy->CreateFilter(slices.data(), 64, &dst);
  return dst.size() < 9 ? -1 : (int)((dst.size() - 1) / 8);
}

inline lc_file_range Range(const FileMetaData* f, int level) {
  const Slice s = f->smallest.Encode(), l = f->largest.Encode();
  lc_file_range r;
  r.smallest = reinterpret_cast<const uint8_t*>(s.data());
  r.smallest_len = (uint32_t)s.size();
  r.largest = reinterpret_cast<const uint8_t*>(l.data());
  r.largest_len = (uint32_t)l.size();
  r.file_size = f->file_size;
  r.level = level;
  return r;
}

// Reads a whole table file into memory.
inline Status ReadWholeFile(Env* env, const std::string& fname, uint64_t size, std::string* out) {
  RandomAccessFile* file = nullptr;
  Status s = env->NewRandomAccessFile(fname, &file);
  if (!s.ok()) return s;
  out->resize(size);
  Slice got;
  s = file->Read(0, size, &got, size ? &(*out)[0] : nullptr);
  if (s.ok() && got.size() != size) s = Status::Corruption("truncated table file", fname);
  if (s.ok() && got.data() != out->data()) memcpy(&(*out)[0], got.data(), size);
  delete file;
  return s;
}

}  // namespace luda_b200_host

Status DBImpl::DoCompactionWork(CompactionState* compact) {
  namespace H = luda_b200_host;
  const uint64_t start_micros = env_->NowMicros();
  int64_t imm_micros = 0;  // Micros spent doing imm_ compactions

  Log(options_.info_log, "Compacting %d@%d + %d@%d files (luda_b200)",
      compact->compaction->num_input_files(0), compact->compaction->level(),
      compact->compaction->num_input_files(1), compact->compaction->level() + 1);

  assert(versions_->NumLevelFiles(compact->compaction->level()) > 0);
  assert(compact->builder == nullptr);
  assert(compact->outfile == nullptr);

  if (snapshots_.empty()) {
    compact->smallest_snapshot = versions_->LastSequence();
  } else {
    compact->smallest_snapshot = snapshots_.oldest()->sequence_number();
  }

  // Release mutex while we're actually doing the compaction work
  mutex_.Unlock();

  Compaction* const c = compact->compaction;
  const int level = c->level();
  Status status;
  lc_engine* engine = H::Engine(&status);
  const int bits_per_key = H::BloomBitsPerKey(options_.filter_policy);
  if (status.ok() && strcmp(user_comparator()->Name(), "leveldb.BytewiseComparator") != 0)
    status = Status::NotSupported("luda_b200: comparator", user_comparator()->Name());
  if (status.ok() && bits_per_key < 0)
    status = Status::NotSupported("luda_b200: filter policy", options_.filter_policy->Name());

  // 1. Input bytes in merge-child order (VersionSet::MakeInputIterator,
  //    db/version_set.cc:1237-1268): one run per level-0 file, one run per
  //    level >= 1.
  std::vector<std::string> bufs;
  std::vector<lc_table> tables;
  std::vector<int32_t> runs;
  for (int which = 0; which < 2 && status.ok(); which++) {
    const std::vector<FileMetaData*>& files = c->inputs_[which];
    if (files.empty()) continue;
    for (size_t i = 0; i < files.size() && status.ok(); i++) {
      bufs.emplace_back();
      status = H::ReadWholeFile(env_, TableFileName(dbname_, files[i]->number),
                                files[i]->file_size, &bufs.back());
    }
    if (level + which == 0) {
      runs.insert(runs.end(), files.size(), 1);
    } else {
      runs.push_back((int32_t)files.size());
    }
  }
  for (const std::string& b : bufs)
    tables.push_back({reinterpret_cast<const uint8_t*>(b.data()), (uint64_t)b.size()});

  // 2. Grandparents (ShouldStopBefore) and every file at levels >= L+2
  //    (IsBaseLevelForKey).
  std::vector<lc_file_range> gp, base;
  for (FileMetaData* f : c->grandparents_) gp.push_back(H::Range(f, level + 2));
  for (int lvl = level + 2; lvl < config::kNumLevels; lvl++)
    for (FileMetaData* f : c->input_version_->files_[lvl]) base.push_back(H::Range(f, lvl));

  lc_job_desc d;
  memset(&d, 0, sizeof(d));
  d.level = level;
  d.n_tables = (int32_t)tables.size();
  d.tables = tables.data();
  d.n_runs = (int32_t)runs.size();
  d.run_table_count = runs.data();
  d.n_grandparents = (int32_t)gp.size();
  d.grandparents = gp.data();
  d.n_base_files = (int32_t)base.size();
  d.base_files = base.data();
  d.smallest_snapshot = compact->smallest_snapshot;
  d.options.block_size = (uint32_t)options_.block_size;
  d.options.restart_interval = (uint32_t)options_.block_restart_interval;
  d.options.bits_per_key = bits_per_key;
  d.options.max_file_size = c->MaxOutputFileSize();
  d.verify_checksums = options_.paranoid_checks ? 1 : 0;

  // 3. The compaction, on the GPU.  While it runs, memtable compactions go
  //    first, as in the reference loop.
  lc_job* job = nullptr;
  if (status.ok()) status = H::ToStatus(lc_job_submit(engine, &d, &job));
  if (status.ok()) {
    while (true) {
      const lc_status st = lc_job_wait(job, 1000000);  // 1 ms slices
      if (st != LC_ERR_TIMEOUT) {
        status = H::ToStatus(st);
        break;
      }
      if (has_imm_.load(std::memory_order_relaxed)) {
        const uint64_t imm_start = env_->NowMicros();
        mutex_.Lock();
        if (imm_ != nullptr) {
          CompactMemTable();
          // Wake up MakeRoomForWrite() if necessary.
          background_work_finished_signal_.SignalAll();
        }
        mutex_.Unlock();
        imm_micros += (env_->NowMicros() - imm_start);
      }
    }
  }
  lc_job_out out;
  memset(&out, 0, sizeof(out));
  if (status.ok()) status = H::ToStatus(lc_job_result(job, &out));
  if (status.ok() && shutting_down_.load(std::memory_order_acquire)) {
    status = Status::IOError("Deleting DB during compaction");
  }

  // 4. The output files, as OpenCompactionOutputFile and
  //    FinishCompactionOutputFile write them.
  for (int i = 0; status.ok() && i < out.n_files; i++) {
    uint64_t file_number;
    {
      mutex_.Lock();
      file_number = versions_->NewFileNumber();
      pending_outputs_.insert(file_number);
      CompactionState::Output o;
      o.number = file_number;
      o.smallest.DecodeFrom(Slice(reinterpret_cast<const char*>(out.key_bytes) +
                                      out.smallest_offset[i], out.smallest_len[i]));
      o.largest.DecodeFrom(Slice(reinterpret_cast<const char*>(out.key_bytes) +
                                     out.largest_offset[i], out.largest_len[i]));
      o.file_size = out.file_size[i];
      compact->outputs.push_back(o);
      mutex_.Unlock();
    }
    const std::string fname = TableFileName(dbname_, file_number);
    WritableFile* file = nullptr;
    status = env_->NewWritableFile(fname, &file);
    if (status.ok()) {
      status = file->Append(Slice(reinterpret_cast<const char*>(out.data) + out.file_offset[i],
                                  out.file_size[i]));
    }
    if (status.ok()) status = file->Sync();
    if (status.ok()) status = file->Close();
    delete file;
    compact->total_bytes += out.file_size[i];
    if (status.ok() && out.file_entries[i] > 0) {
      // Verify that the table is usable
      Iterator* iter = table_cache_->NewIterator(ReadOptions(), file_number, out.file_size[i]);
      status = iter->status();
      delete iter;
      if (status.ok()) {
        Log(options_.info_log, "Generated table #%llu@%d: %lld keys, %lld bytes",
            (unsigned long long)file_number, level, (unsigned long long)out.file_entries[i],
            (unsigned long long)out.file_size[i]);
      }
    }
  }
  if (job != nullptr) lc_job_release(job);
  if (status.ok()) H::ServedCount()++;

  CompactionStats stats;
  stats.micros = env_->NowMicros() - start_micros - imm_micros;
  for (int which = 0; which < 2; which++) {
    for (int i = 0; i < compact->compaction->num_input_files(which); i++) {
      stats.bytes_read += compact->compaction->input(which, i)->file_size;
    }
  }
  for (size_t i = 0; i < compact->outputs.size(); i++) {
    stats.bytes_written += compact->outputs[i].file_size;
  }

  mutex_.Lock();
  stats_[compact->compaction->level() + 1].Add(stats);

  if (status.ok()) {
    status = InstallCompactionResults(compact);
  }
  if (!status.ok()) {
    RecordBackgroundError(status);
  }
  VersionSet::LevelSummaryStorage tmp;
  Log(options_.info_log, "compacted to: %s", versions_->LevelSummary(&tmp));
  return status;
}

// Compactions this process's DBs have run through the engine (diagnostics).
extern "C" uint64_t luda_b200_host_compactions_served() {
  return luda_b200_host::ServedCount().load();
}
