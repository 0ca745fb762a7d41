// Test infrastructure, not product code.
//
// One seeded workload driven through the public leveldb::DB API of whichever
// LevelDB it is linked with: the reference's own build with its CPU
// DBImpl::DoCompactionWork (db_scenario_cpu), or the same reference sources
// with DoCompactionWork replaced by the luda_b200 drop-in
// (db_scenario_luda_b200; see oracle/Makefile, target dropin).
//
//   db_scenario <db dir> <seed>
//
// Writes five batches of puts and deletes (16-byte zero-padded decimal keys of
// uniform ints in [0, 2^20), as db/db_bench.cc:729 makes them, 100-byte values,
// ~10% rewrites, ~2% deletions), flushing each memtable to a table
// (DBImpl::TEST_CompactMemTable, db/db_impl.cc:756) and compacting level 0
// into level 1 and level 1 into level 2 with DBImpl::TEST_CompactRange
// (db/db_impl.cc:725-779), with a snapshot held across the later batches.
// Then reads everything back through an iterator, through Get and through
// the snapshot and compares it with an in-memory model of the writes.  Prints
// one JSON line; the caller compares the table files of the two builds.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "db/db_impl.h"
#include "leveldb/db.h"
#include "leveldb/filter_policy.h"
#include "leveldb/options.h"
#include "leveldb/write_batch.h"

// Compactions served by the drop-in (defined in its build only).
extern "C" uint64_t luda_b200_host_compactions_served() __attribute__((weak));

namespace {

using namespace leveldb;

struct Rng {
  uint64_t s;
  uint64_t next() {  // splitmix64
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
};

std::string Key(uint64_t id) {
  char buf[32];
  snprintf(buf, sizeof(buf), "%016d", (int)id);
  return std::string(buf, 16);
}

int Fail(const std::string& what, const Status& s) {
  printf("{\"ok\": false, \"status\": \"%s: %s\"}\n", what.c_str(), s.ToString().c_str());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <db dir> <seed>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  Rng rng{(uint64_t)strtoull(argv[2], nullptr, 10)};
  const FilterPolicy* policy = NewBloomFilterPolicy(10);
  Options opt;
  opt.create_if_missing = true;
  opt.write_buffer_size = 64 << 20;  // flushes happen only where the scenario asks
  opt.block_size = 4096;
  opt.block_restart_interval = 16;
  opt.compression = kNoCompression;
  opt.filter_policy = policy;
  opt.max_file_size = 1 << 20;
  DestroyDB(dir, opt);
  DB* db = nullptr;
  Status s = DB::Open(opt, dir, &db);
  if (!s.ok()) return Fail("open", s);
  DBImpl* impl = reinterpret_cast<DBImpl*>(db);

  std::map<std::string, std::string> model;
  std::vector<uint64_t> written;
  std::map<std::string, std::string> at_snapshot;
  const Snapshot* snap = nullptr;
  const int kBatches = 5, kPerBatch = 16000;
  for (int b = 0; b < kBatches; b++) {
    WriteBatch wb;
    for (int i = 0; i < kPerBatch; i++) {
      const uint64_t r = rng.next();
      uint64_t id = r % (1u << 20);
      if (!written.empty() && (r >> 40) % 10 == 0) id = written[(r >> 20) % written.size()];
      const std::string k = Key(id);
      if (!written.empty() && (r >> 48) % 50 == 0) {
        wb.Delete(k);
        model.erase(k);
      } else {
        std::string v(100, '\0');
        for (int j = 0; j < 100; j += 8) {
          const uint64_t x = rng.next();
          for (int t = 0; t < 8 && j + t < 100; t++) v[j + t] = (char)(x >> (8 * t));
        }
        wb.Put(k, v);
        model[k] = v;
        written.push_back(id);
      }
      if (wb.ApproximateSize() > (1 << 20)) {
        s = db->Write(WriteOptions(), &wb);
        if (!s.ok()) return Fail("write", s);
        wb.Clear();
      }
    }
    s = db->Write(WriteOptions(), &wb);
    if (!s.ok()) return Fail("write", s);
    s = impl->TEST_CompactMemTable();
    if (!s.ok()) return Fail("flush", s);
    if (b == 1) {
      snap = db->GetSnapshot();
      at_snapshot = model;
    }
    if (b == 2) impl->TEST_CompactRange(0, nullptr, nullptr);
  }
  impl->TEST_CompactRange(0, nullptr, nullptr);
  impl->TEST_CompactRange(1, nullptr, nullptr);

  int levels[7];
  for (int l = 0; l < 7; l++) {
    std::string v;
    db->GetProperty("leveldb.num-files-at-level" + std::to_string(l), &v);
    levels[l] = atoi(v.c_str());
  }

  // everything back, compared with the model
  uint64_t mismatches = 0, entries = 0;
  Iterator* it = db->NewIterator(ReadOptions());
  auto m = model.begin();
  for (it->SeekToFirst(); it->Valid(); it->Next(), entries++) {
    if (m == model.end() || it->key().ToString() != m->first ||
        it->value().ToString() != m->second)
      mismatches++;
    if (m != model.end()) ++m;
  }
  if (m != model.end()) mismatches++;
  if (!it->status().ok()) return Fail("iterator", it->status());
  delete it;
  uint64_t get_mismatches = 0;
  for (int i = 0; i < 4000; i++) {
    const std::string k = Key(rng.next() % (1u << 20));
    std::string v;
    s = db->Get(ReadOptions(), k, &v);
    auto f = model.find(k);
    if (f == model.end() ? !s.IsNotFound() : (!s.ok() || v != f->second)) get_mismatches++;
  }
  uint64_t snap_mismatches = 0;
  {
    ReadOptions ro;
    ro.snapshot = snap;
    Iterator* si = db->NewIterator(ro);
    auto e = at_snapshot.begin();
    for (si->SeekToFirst(); si->Valid(); si->Next()) {
      if (e == at_snapshot.end() || si->key().ToString() != e->first ||
          si->value().ToString() != e->second)
        snap_mismatches++;
      if (e != at_snapshot.end()) ++e;
    }
    if (e != at_snapshot.end()) snap_mismatches++;
    delete si;
  }
  db->ReleaseSnapshot(snap);
  std::string stats;
  db->GetProperty("leveldb.stats", &stats);
  const long long served =
      luda_b200_host_compactions_served ? (long long)luda_b200_host_compactions_served() : -1;
  delete db;
  delete policy;
  printf("{\"ok\": true, \"entries\": %" PRIu64 ", \"model_entries\": %zu, \"mismatches\": %" PRIu64
         ", \"get_mismatches\": %" PRIu64 ", \"snapshot_mismatches\": %" PRIu64
         ", \"levels\": [%d, %d, %d, %d, %d, %d, %d], \"served\": %lld}\n",
         entries, model.size(), mismatches, get_mismatches, snap_mismatches, levels[0], levels[1],
         levels[2], levels[3], levels[4], levels[5], levels[6], served);
  return 0;
}
