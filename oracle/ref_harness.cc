// Test infrastructure, not product code.
//
// Drives the reference LevelDB (LUDA fork) CPU compaction synchronously so that
// its outputs can serve as the byte-exact oracle for the GPU engine, and so that
// the reference's own CPU path can be timed as the baseline.  Compiled by
// oracle/Makefile into oracle/_ref/libluda_ref.so directly from the reference
// sources; nothing in the product links against it.
//
// The translation unit includes a copy of db/db_impl.cc whose only change is
// GPU_ACCELERATE set to 0 (db/db_impl.cc:44), which selects the CPU
// DBImpl::DoCompactionWork (db/db_impl.cc:1060-1224).  CompactionState is a
// struct private to that file (db/db_impl.cc:195-227), so the harness must live
// in the same translation unit.
//
// Flow of one job (mirrors what DBImpl::BackgroundCompaction does around
// DoCompactionWork, db/db_impl.cc:854-951, but synchronously):
//   1. open a DB on an in-memory Env (helpers/memenv/memenv.cc);
//   2. write the input tables as files and install them, plus metadata-only
//      files for deeper levels, with one VersionEdit + LogAndApply
//      (db/version_set.cc:801);
//   3. set LastSequence and create the snapshots (db/snapshot.h:57);
//   4. build the Compaction exactly as VersionSet::SetupOtherInputs does for
//      grandparents (db/version_set.cc:1405-1463), with inputs_[0]/inputs_[1]
//      = all files of level L / L+1 in the version's order;
//   5. call DoCompactionWork with mutex_ held (it unlocks for the work and
//      re-locks before InstallCompactionResults);
//   6. read the produced files back from the Env.

#include REF_DB_IMPL_CC

#include <chrono>
#include <thread>

#include "helpers/memenv/memenv.h"
#include "leveldb/filter_policy.h"
#include "leveldb/table.h"
#include "table/block_builder.h"
#include "table/filter_block.h"
#include "util/crc32c.h"
#include "util/hash.h"

extern "C" {

typedef struct {
  const uint8_t* data;  // table bytes; NULL for a metadata-only file
  uint64_t size;        // file_size recorded in the version
  int32_t level;
  const uint8_t* smallest;  // internal key
  uint32_t smallest_len;
  const uint8_t* largest;  // internal key
  uint32_t largest_len;
} ref_file;

typedef struct {
  int32_t level;
  int32_t n_files;
  const ref_file* files;
  int32_t n_snapshots;
  const uint64_t* snapshots;
  uint64_t last_sequence;
  uint32_t block_size;
  uint32_t restart_interval;
  int32_t bits_per_key;  // <= 0: no filter policy
  uint64_t max_file_size;
} ref_job;

typedef struct {
  std::string bytes;
  std::string smallest;
  std::string largest;
  uint64_t number;
} ref_out_file;

typedef struct {
  int status;  // 0 ok, else error
  std::string message;
  std::vector<ref_out_file> files;
  double seconds;  // wall time of DoCompactionWork, entry to return
} ref_result;

typedef struct {
  std::string bytes;
} ref_buf;

}  // extern "C"

namespace {

using namespace leveldb;

Options MakeOptions(const ref_job* job, Env* env, const FilterPolicy* policy) {
  Options opt;
  opt.env = env;
  opt.create_if_missing = true;
  opt.block_size = job->block_size;
  opt.block_restart_interval = job->restart_interval;
  opt.compression = kNoCompression;
  opt.filter_policy = policy;
  opt.max_file_size = job->max_file_size;
  return opt;
}

void RunJob(const ref_job* job, ref_result* res, const std::string& dbname) {
  Env* env = NewMemEnv(Env::Default());
  const FilterPolicy* policy =
      job->bits_per_key > 0 ? NewBloomFilterPolicy(job->bits_per_key) : nullptr;
  Options opt = MakeOptions(job, env, policy);
  DB* db = nullptr;
  Status s = DB::Open(opt, dbname, &db);
  if (!s.ok()) {
    res->status = 1;
    res->message = s.ToString();
    delete env;
    delete policy;
    return;
  }
  DBImpl* impl = reinterpret_cast<DBImpl*>(db);

  VersionEdit edit;
  impl->mutex_.Lock();
  std::vector<uint64_t> numbers(job->n_files);
  for (int i = 0; i < job->n_files; i++) numbers[i] = impl->versions_->NewFileNumber();
  impl->mutex_.Unlock();

  for (int i = 0; i < job->n_files && s.ok(); i++) {
    const ref_file& f = job->files[i];
    if (f.data != nullptr) {
      WritableFile* wf = nullptr;
      s = env->NewWritableFile(TableFileName(dbname, numbers[i]), &wf);
      if (s.ok()) s = wf->Append(Slice(reinterpret_cast<const char*>(f.data), f.size));
      if (s.ok()) s = wf->Close();
      delete wf;
    }
    InternalKey smallest, largest;
    smallest.DecodeFrom(Slice(reinterpret_cast<const char*>(f.smallest), f.smallest_len));
    largest.DecodeFrom(Slice(reinterpret_cast<const char*>(f.largest), f.largest_len));
    edit.AddFile(f.level, numbers[i], f.size, smallest, largest);
  }

  impl->mutex_.Lock();
  if (s.ok()) {
    impl->versions_->SetLastSequence(job->last_sequence);
    s = impl->versions_->LogAndApply(&edit, &impl->mutex_);
  }
  for (int i = 0; i < job->n_snapshots; i++) impl->snapshots_.New(job->snapshots[i]);

  Compaction* c = nullptr;
  DBImpl::CompactionState* compact = nullptr;
  if (s.ok()) {
    const int level = job->level;
    c = new Compaction(impl->versions_->options_, level);
    c->input_version_ = impl->versions_->current();
    c->input_version_->Ref();
    c->inputs_[0] = c->input_version_->files_[level];
    c->inputs_[1] = c->input_version_->files_[level + 1];
    InternalKey all_start, all_limit;
    impl->versions_->GetRange2(c->inputs_[0], c->inputs_[1], &all_start, &all_limit);
    if (level + 2 < config::kNumLevels) {
      c->input_version_->GetOverlappingInputs(level + 2, &all_start, &all_limit,
                                              &c->grandparents_);
    }
    compact = new DBImpl::CompactionState(c);
    auto t0 = std::chrono::steady_clock::now();
    s = impl->DoCompactionWork(compact);  // returns with mutex_ held
    auto t1 = std::chrono::steady_clock::now();
    res->seconds = std::chrono::duration<double>(t1 - t0).count();
  }
  if (s.ok()) {
    for (size_t i = 0; i < compact->outputs.size(); i++) {
      const auto& out = compact->outputs[i];
      ref_out_file of;
      of.number = out.number;
      of.smallest = out.smallest.Encode().ToString();
      of.largest = out.largest.Encode().ToString();
      Status rs = ReadFileToString(env, TableFileName(dbname, out.number), &of.bytes);
      if (!rs.ok()) s = rs;
      res->files.push_back(std::move(of));
    }
  }
  if (compact != nullptr) impl->CleanupCompaction(compact);
  if (c != nullptr) {
    c->ReleaseInputs();
    delete c;
  }
  impl->mutex_.Unlock();
  res->status = s.ok() ? 0 : 2;
  if (!s.ok()) res->message = s.ToString();
  delete db;
  delete env;
  delete policy;
}

// In-memory sink for TableBuilder.
class StringSink : public WritableFile {
 public:
  std::string contents;
  Status Append(const Slice& data) override {
    contents.append(data.data(), data.size());
    return Status::OK();
  }
  Status Close() override { return Status::OK(); }
  Status Flush() override { return Status::OK(); }
  Status Sync() override { return Status::OK(); }
};

class StringSource : public RandomAccessFile {
 public:
  explicit StringSource(const std::string& s) : contents_(s) {}
  Status Read(uint64_t offset, size_t n, Slice* result, char* scratch) const override {
    if (offset >= contents_.size()) return Status::InvalidArgument("bad offset");
    if (offset + n > contents_.size()) n = contents_.size() - offset;
    memcpy(scratch, contents_.data() + offset, n);
    *result = Slice(scratch, n);
    return Status::OK();
  }

 private:
  std::string contents_;
};

}  // namespace

extern "C" {

// Runs one compaction through the reference's CPU DoCompactionWork.
ref_result* ref_compact(const ref_job* job) {
  ref_result* res = new ref_result();
  res->status = 0;
  res->seconds = 0;
  static std::atomic<int> counter{0};
  RunJob(job, res, "/refdb" + std::to_string(counter.fetch_add(1)));
  return res;
}

// Runs the same job on n_threads threads at once (each its own DB), returns
// the wall seconds of the slowest DoCompactionWork; used for the all-cores
// CPU baseline.
double ref_compact_parallel(const ref_job* job, int n_threads, int* status) {
  std::vector<ref_result> results(n_threads);
  std::vector<std::thread> threads;
  static std::atomic<int> counter{0};
  auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n_threads; i++) {
    int id = counter.fetch_add(1);
    threads.emplace_back([job, &results, i, id]() {
      results[i].status = 0;
      RunJob(job, &results[i], "/refpar" + std::to_string(id));
    });
  }
  for (auto& t : threads) t.join();
  auto t1 = std::chrono::steady_clock::now();
  *status = 0;
  for (auto& r : results)
    if (r.status != 0) *status = r.status;
  return std::chrono::duration<double>(t1 - t0).count();
}

int ref_result_status(const ref_result* r) { return r->status; }
const char* ref_result_message(const ref_result* r) { return r->message.c_str(); }
double ref_result_seconds(const ref_result* r) { return r->seconds; }
int ref_result_nfiles(const ref_result* r) { return (int)r->files.size(); }
const uint8_t* ref_result_file(const ref_result* r, int i, uint64_t* len) {
  *len = r->files[i].bytes.size();
  return reinterpret_cast<const uint8_t*>(r->files[i].bytes.data());
}
const uint8_t* ref_result_smallest(const ref_result* r, int i, uint32_t* len) {
  *len = r->files[i].smallest.size();
  return reinterpret_cast<const uint8_t*>(r->files[i].smallest.data());
}
const uint8_t* ref_result_largest(const ref_result* r, int i, uint32_t* len) {
  *len = r->files[i].largest.size();
  return reinterpret_cast<const uint8_t*>(r->files[i].largest.data());
}
void ref_result_free(ref_result* r) { delete r; }

const uint8_t* ref_buf_data(const ref_buf* b, uint64_t* len) {
  *len = b->bytes.size();
  return reinterpret_cast<const uint8_t*>(b->bytes.data());
}
void ref_buf_free(ref_buf* b) { delete b; }

// TableBuilder over n sorted internal keys (concatenated, with n+1 offsets)
// and values: the reference's own flush encoder (db/builder.cc:17-60 feeds
// TableBuilder the same way).
ref_buf* ref_build_table(uint32_t block_size, uint32_t restart_interval, int bits_per_key,
                         int64_t n, const uint8_t* keys, const uint64_t* key_offs,
                         const uint8_t* vals, const uint64_t* val_offs) {
  InternalKeyComparator icmp(BytewiseComparator());
  const FilterPolicy* policy = bits_per_key > 0 ? NewBloomFilterPolicy(bits_per_key) : nullptr;
  InternalFilterPolicy ipolicy(policy);
  Options opt;
  opt.comparator = &icmp;
  opt.filter_policy = policy ? &ipolicy : nullptr;
  opt.block_size = block_size;
  opt.block_restart_interval = restart_interval;
  opt.compression = kNoCompression;
  StringSink sink;
  TableBuilder tb(opt, &sink);
  for (int64_t i = 0; i < n; i++) {
    tb.Add(Slice(reinterpret_cast<const char*>(keys) + key_offs[i], key_offs[i + 1] - key_offs[i]),
           Slice(reinterpret_cast<const char*>(vals) + val_offs[i], val_offs[i + 1] - val_offs[i]));
  }
  tb.Finish();
  ref_buf* b = new ref_buf();
  b->bytes = std::move(sink.contents);
  delete policy;
  return b;
}

// Reads every entry of a table through the unchanged Table iterator
// (table/table.cc:38 Open, two-level iterator over the index).  Output is
// a flat record stream: fixed32 klen, key, fixed32 vlen, value.  status<0 on
// error.
ref_buf* ref_read_table(const uint8_t* data, uint64_t size, int bits_per_key, int* status) {
  InternalKeyComparator icmp(BytewiseComparator());
  const FilterPolicy* policy = bits_per_key > 0 ? NewBloomFilterPolicy(bits_per_key) : nullptr;
  InternalFilterPolicy ipolicy(policy);
  Options opt;
  opt.comparator = &icmp;
  opt.filter_policy = policy ? &ipolicy : nullptr;
  StringSource* src = new StringSource(std::string(reinterpret_cast<const char*>(data), size));
  Table* table = nullptr;
  Status s = Table::Open(opt, src, size, &table);
  ref_buf* b = new ref_buf();
  *status = 0;
  if (!s.ok()) {
    *status = -1;
    b->bytes = s.ToString();
    delete src;
    delete policy;
    return b;
  }
  ReadOptions ro;
  ro.verify_checksums = true;
  Iterator* it = table->NewIterator(ro);
  for (it->SeekToFirst(); it->Valid(); it->Next()) {
    PutFixed32(&b->bytes, it->key().size());
    b->bytes.append(it->key().data(), it->key().size());
    PutFixed32(&b->bytes, it->value().size());
    b->bytes.append(it->value().data(), it->value().size());
  }
  if (!it->status().ok()) *status = -2;
  delete it;
  delete table;
  delete src;
  delete policy;
  return b;
}

// Primitive known-answer helpers: the reference's own functions.
uint32_t ref_crc32c(const uint8_t* data, uint64_t n) {
  return leveldb::crc32c::Value(reinterpret_cast<const char*>(data), n);
}
uint32_t ref_crc32c_mask(uint32_t crc) { return leveldb::crc32c::Mask(crc); }
uint32_t ref_hash(const uint8_t* data, uint64_t n, uint32_t seed) {
  return leveldb::Hash(reinterpret_cast<const char*>(data), n, seed);
}

// BloomFilterPolicy::CreateFilter over user keys (util/bloom.cc:28-54).
ref_buf* ref_bloom(int bits_per_key, int n, const uint8_t* keys, const uint64_t* key_offs) {
  const FilterPolicy* policy = NewBloomFilterPolicy(bits_per_key);
  std::vector<Slice> ks;
  for (int i = 0; i < n; i++)
    ks.emplace_back(reinterpret_cast<const char*>(keys) + key_offs[i], key_offs[i + 1] - key_offs[i]);
  ref_buf* b = new ref_buf();
  policy->CreateFilter(ks.data(), n, &b->bytes);
  delete policy;
  return b;
}

// InternalKeyComparator separator / successor (db/dbformat.cc:69-101).
ref_buf* ref_separator(const uint8_t* a, uint32_t alen, const uint8_t* b, uint32_t blen) {
  InternalKeyComparator icmp(BytewiseComparator());
  ref_buf* r = new ref_buf();
  r->bytes.assign(reinterpret_cast<const char*>(a), alen);
  icmp.FindShortestSeparator(&r->bytes, Slice(reinterpret_cast<const char*>(b), blen));
  return r;
}
ref_buf* ref_successor(const uint8_t* a, uint32_t alen) {
  InternalKeyComparator icmp(BytewiseComparator());
  ref_buf* r = new ref_buf();
  r->bytes.assign(reinterpret_cast<const char*>(a), alen);
  icmp.FindShortSuccessor(&r->bytes);
  return r;
}

}  // extern "C"
