/* Test infrastructure, not product code.
 *
 * CPU restatement of the reference's LSM compaction path (LevelDB 1.22 as
 * modified by LUDA), used only as the checker for the GPU engine: by tests/,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  Parity of
 * this restatement is pinned against the reference itself (oracle/_ref, built
 * from the reference sources) and against the reference's known-answer vectors.
 */
#ifndef LSM_ORACLE_H_
#define LSM_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  const uint8_t* data;
  uint64_t size;
} lo_table;

/* A file at a level >= L+2: only its key range and size matter. */
typedef struct {
  const uint8_t* smallest; /* internal key */
  uint32_t smallest_len;
  const uint8_t* largest; /* internal key */
  uint32_t largest_len;
  uint64_t file_size;
  int32_t level;
} lo_file_range;

typedef struct {
  int32_t level;
  int32_t n_tables;
  const lo_table* tables; /* run-major, runs in merge-child order */
  int32_t n_runs;
  const int32_t* run_table_count;
  int32_t n_grandparents; /* Compaction::grandparents_ in key order */
  const lo_file_range* grandparents;
  int32_t n_base_files; /* every file at levels >= L+2, each level in key order */
  const lo_file_range* base_files;
  uint64_t smallest_snapshot;
  uint32_t block_size;
  uint32_t restart_interval;
  int32_t bits_per_key; /* <= 0: no filter block */
  uint64_t max_file_size;
} lo_job;

typedef struct lo_result lo_result;
typedef struct lo_buf lo_buf;

/* Compaction (db/db_impl.cc:1060-1224).  *status: 0 ok, 1 bad argument,
 * 2 corrupt input. */
lo_result* lo_compact(const lo_job* job, int* status);
int lo_result_nfiles(const lo_result* r);
const uint8_t* lo_result_file(const lo_result* r, int i, uint64_t* len);
const uint8_t* lo_result_smallest(const lo_result* r, int i, uint32_t* len);
const uint8_t* lo_result_largest(const lo_result* r, int i, uint32_t* len);
uint64_t lo_result_entries(const lo_result* r, int i);
void lo_result_free(lo_result* r);

/* TableBuilder over sorted internal keys (table/table_builder.cc). */
lo_buf* lo_build_table(uint32_t block_size, uint32_t restart_interval, int bits_per_key,
                       int64_t n, const uint8_t* keys, const uint64_t* key_offs,
                       const uint8_t* vals, const uint64_t* val_offs);
/* Decodes every entry of a table: fixed32 klen, key, fixed32 vlen, value. */
lo_buf* lo_read_table(const uint8_t* data, uint64_t size, int* status);
const uint8_t* lo_buf_data(const lo_buf* b, uint64_t* len);
void lo_buf_free(lo_buf* b);

/* Primitives. */
uint32_t lo_crc32c_extend(uint32_t crc, const uint8_t* data, uint64_t n);
uint32_t lo_crc32c_mask(uint32_t crc);
uint32_t lo_hash(const uint8_t* data, uint64_t n, uint32_t seed);
lo_buf* lo_bloom(int bits_per_key, int n, const uint8_t* keys, const uint64_t* key_offs);
lo_buf* lo_separator(const uint8_t* a, uint32_t alen, const uint8_t* b, uint32_t blen);
lo_buf* lo_successor(const uint8_t* a, uint32_t alen);

#ifdef __cplusplus
}
#endif
#endif
