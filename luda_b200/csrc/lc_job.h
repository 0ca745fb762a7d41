// Device-side state of one compaction job, shared by the host orchestration
// (lc_engine.cu) and the kernels.  All arrays live in HBM; the struct itself is
// passed to kernels by value.
//
// Data layout in HBM (one job):
//   in        input tables back to back, each starting on a 16-byte boundary
//   tables    per input table: offset in `in`, size, run index
//   blocks    per input data block: offset in `in`, size, entry/key bases
//   entries   per decoded entry (structure of arrays, input order):
//               koff/klen  internal key in the key arena `keys`
//               voff/vlen  value bytes, left in place inside `in`
//               pfx        first 8 user-key bytes, big endian (compare fast path)
//   merged    entry ids in merge order; kept ids after the drop rule
//   per kept entry: restart/compressed sizes, shared prefix, block-start flag
//   per output block / filter group / file: sizes, offsets, separators
//   out       all output files back to back
#pragma once
#include <stdint.h>

namespace lc {

// Job error codes written to Counters::error by kernels (first error wins).
enum : uint32_t {
  kErrNone = 0,
  kErrBadFooter = 1,      // magic or footer handles invalid
  kErrBadIndex = 2,       // index block malformed
  kErrBadBlock = 3,       // data block trailer / restart array malformed
  kErrBadEntry = 4,       // entry header or lengths out of range
  kErrShortKey = 5,       // internal key shorter than 8 bytes
  kErrArenaOverflow = 6,  // decoded keys exceed the arena capacity
  kErrLimit = 7,          // an engine limit was exceeded
  kErrRetryExact = 8,     // the single-pass decode's bounded key arena (or key length
                          // bound) was too small: the host reruns the job with counting
  kErrChecksum = 9,       // a data block's stored CRC32C does not match its contents
  kErrUnsorted = 10,      // a merge child's entries are not in internal-key order
};

struct Counters {
  uint32_t error;
  uint32_t error_detail;
  uint32_t max_klen;
  uint32_t max_jump;
  uint64_t n_blocks_in;
  uint64_t n_entries_in;
  uint64_t key_bytes_in;
  uint64_t n_kept;
  uint64_t n_blocks_out;
  uint64_t bytes_out;
  uint32_t n_triggers;
  uint32_t n_files;
  uint32_t n_groups;
  uint32_t pad;
  uint64_t kept_key_bytes;    // internal-key bytes of the survivors
  uint64_t kept_value_bytes;  // value bytes of the survivors
  uint64_t key_cursor;        // key bytes of the decoded entries (the scan of their lengths)
  uint32_t key_skip;          // user-key bytes every input key shares (prefixes start after them)
  uint32_t pad2;
  uint64_t key_total;         // decoded key bytes, summed by the decode's first pass
};

struct TableDesc {
  uint64_t off;   // in `in`
  uint64_t size;
  uint32_t run;
  uint32_t cached;  // 1: read from its decoded form (JobDev::dec_runs[t]), not parsed
};

// The decoded entries of one table, kept by the job that wrote it: entry j
// has the key keys[kcum[j], kcum[j+1]) and its value at byte vpos[j] of the
// table, vlen[j] bytes long; pfx and tag as e_pfx / e_tag.
struct DecRun {
  uint64_t n;
  const uint8_t* keys;
  const uint64_t* kcum;  // n + 1, absolute in `keys`
  const uint32_t* vlen;
  const uint32_t* vpos;
  const uint64_t* pfx;
  const uint64_t* tag;
};

// Entries per pseudo block of a table read from its decoded form.
constexpr uint32_t kDecRunBlock = 256;
// blk_size of a pseudo block; its blk_off is (table << 32) | first entry.
constexpr uint32_t kPseudoBlock = 0xffffffffu;

struct FileOut {       // per output file
  uint64_t out_off;    // offset of the file in `out`
  uint64_t size;       // file size
  uint64_t data_bytes; // data region (blocks + trailers)
  uint64_t filter_off, filter_size;   // filter block handle (within file)
  uint64_t meta_off, meta_size;       // metaindex block handle
  uint64_t index_off, index_size;     // index block handle
  uint64_t first_kept, end_kept;      // kept entries [first, end)
  uint32_t first_block, end_block;    // output blocks [first, end)
  uint32_t n_filters;                 // filter offsets in the filter block
  uint32_t crc_acc[3];                // raw CRC32C registers of the filter, metaindex and
                                      // index blocks, xored together from pieces
};

struct JobDev {
  // options
  uint32_t block_size;
  uint32_t restart_interval;
  int32_t bits_per_key;  // <= 0: no filter
  uint32_t bloom_k;
  uint32_t verify_checksums;  // check every input data block's trailer CRC
  uint64_t max_file_size;
  uint64_t smallest_snapshot;
  int64_t max_gp_overlap;  // 10 * max_file_size

  // input
  const uint8_t* in;
  uint64_t in_size;
  const uint8_t* in_end;  // end of memory that may be read with 16-byte loads
  const TableDesc* tables;
  const DecRun* dec_runs;    // per table (n = 0 where the table is parsed)
  uint32_t n_tables;
  uint32_t n_runs;
  const uint64_t* run_entry_begin;  // filled after decode: entries of run r are
                                    // [run_entry_begin[r], run_entry_begin[r+1])
  uint64_t* run_entry_begin_w;

  // grandparents: largest internal keys (packed) and sizes, key order
  uint32_t n_gp;
  const uint8_t* gp_keys;
  const uint64_t* gp_key_off;   // n_gp + 1
  const uint64_t* gp_prefix;    // n_gp + 1, prefix sums of file sizes
  uint64_t* gp_upfx;            // n_gp: 8 user-key bytes of each largest key after the
                                // job's common prefix, big endian (k_key_skip)
  uint8_t* gp_mode;             // n_gp: 0 compare by prefix then key; 1 every entry sorts
                                // after the grandparent; 2 every entry sorts before it
  // base-level files: user-key ranges per level >= L+2
  uint32_t n_base_levels;
  const uint32_t* base_level_begin;  // n_base_levels + 1, into the file list
  const uint8_t* base_keys;
  const uint64_t* base_small_off;    // per file: smallest user key [off, off+len)
  const uint32_t* base_small_len;
  const uint64_t* base_large_off;
  const uint32_t* base_large_len;

  Counters* ctr;

  // input blocks
  uint32_t* tbl_nblocks;     // n_tables
  uint32_t* tbl_unit;        // n_tables: 1 when every index restart run holds one entry
  uint64_t* tbl_block_base;  // n_tables + 1
  uint64_t* blk_off;         // cap_blocks_in
  uint32_t* blk_size;
  uint32_t* blk_run;         // merge child of the block
  uint32_t* blk_nent;        // entries per block
  uint64_t* blk_ent_base;    // cap_blocks_in + 1
  uint64_t* blk_kbytes;      // key bytes per block
  uint64_t* blk_key_base;    // cap_blocks_in + 1
  uint64_t cap_blocks_in;

  // entries (input order)
  uint8_t* keys;             // key arena
  uint64_t cap_key_bytes;
  uint4* e_rec;              // per entry: decode record (pass 1 -> pass 2)
  uint32_t dec_group;        // data blocks per warp in the decode's first pass
  uint32_t* e_koff;
  uint32_t* e_klen;
  uint32_t* e_voff;
  uint32_t* e_vlen;
  uint64_t* e_pfx;           // 8 user-key bytes after the key_skip common bytes, big endian
  uint64_t* e_tag;           // the key's last 8 bytes: (sequence << 8) | type
  uint64_t cap_entries;

  // merge
  uint32_t* m_ids;           // merged order (holds the result after the last round)
  uint32_t* m_tmp;           // the other buffer of the ping-pong
  uint64_t* m_pfx;           // e_pfx of m_ids, in merged order (result after the last round)
  uint64_t* m_pfx_tmp;       // the other buffer of the ping-pong
  uint64_t* m_tag;           // e_tag of m_ids, in merged order (result after the last round)
  uint64_t* m_tag_tmp;       // the other buffer of the ping-pong
  uint32_t* m_split;         // per merge tile: first-group elements before the tile
  uint32_t cap_merge_tiles;  // capacity of m_split
  uint8_t* keep;             // per merged position
  uint32_t* gp_idx;          // per merged position: grandparents passed
  uint32_t* kept_pos;        // exclusive scan of keep (n+1)
  uint32_t* triggers;        // merged positions where ShouldStopBefore fires
  uint32_t cap_triggers;

  // kept entries
  uint32_t* k_koff;          // survivors, in output order: key offset in the arena,
  uint32_t* k_klen;          // key length,
  uint32_t* k_voff;          // value offset in `in`,
  uint32_t* k_vlen;          // value length (gathered once from the entry arrays)

  // the survivors' decoded form, kept for later jobs (keep_decoded; else null)
  uint8_t* dec_keys;         // keys in survivor order
  uint64_t* dec_kcum;        // n_kept + 1: key offsets in dec_keys
  uint32_t* dec_vlen;
  uint32_t* dec_vpos;        // value offset within its output file (by k_encode_blocks)
  uint64_t* dec_pfx;
  uint64_t* dec_tag;
  uint32_t* k_a;             // size as a restart entry
  uint32_t* k_b;             // size as a prefix-compressed entry
  uint32_t* k_shared;        // shared prefix with the previous kept key
  uint8_t* k_forced;         // a block (and file) must start here
  uint32_t* k_next;          // first entry of the next block if a block starts here
  uint8_t* k_bstart;         // block starts here
  uint32_t* k_block;         // exclusive scan of k_bstart (n+1)

  // chain resolution
  uint32_t chunk;            // entries per chunk
  uint32_t* chunk_table;     // per chunk: exit for each window entry
  uint32_t* chunk_entry;     // per chunk: resolved entry point
  uint32_t* group_table;     // per group of kChainGroup chunks: exit for each window entry
  uint32_t window;           // table width
  uint32_t chain_smem_words; // shared-memory words for staging the chunk tables
  uint32_t reserve_keys;     // 1: decode reserves key-arena space per block (single
                             // pass, restart counts only); 0: blk_key_base from counting
  uint32_t max_key_len;      // 1: longest key the single-pass layout allows

  // output blocks
  uint32_t* b_first;         // first kept entry of block (cap_blocks_out + 1)
  uint32_t* b_size;          // block contents size (without trailer)
  uint64_t* b_cum;           // prefix of (b_size + 5), cap_blocks_out + 1
  uint32_t* b_file;          // file of block
  uint64_t* b_off;           // block offset within its file
  uint32_t* b_isize;         // index entry size
  uint64_t* b_icum;          // prefix of index entry sizes
  uint32_t* b_sep;           // index key: 0xffffffff = last key unchanged, else the
                             // shortened user-key length minus one (byte at that
                             // position is incremented, then the seek tag follows)
  uint32_t* b_ilen;          // index key length
  uint32_t* b_gbytes;        // filter group bytes (nonzero at group starts)
  uint64_t* b_gcum;          // prefix of b_gbytes
  uint32_t* b_gkeys;         // keys in the group (at group starts)
  uint32_t* b_fnext;         // first block of the next file if a file starts here
  uint32_t* t_blocks;        // output block starting at each grandparent cut
  uint32_t* t_kept;          // survivor position of each grandparent cut (ascending)
  uint64_t* k_pb;            // n_kept + 1: prefix sums of k_b (block size estimates)
  uint64_t cap_blocks_out;

  // files
  FileOut* files;
  uint32_t cap_files;
  uint8_t* out;
  uint64_t cap_out;

  // scratch of the batched kernels
  uint32_t* gp_first;        // per grandparent count g: first merged position reaching g
  uint32_t* tmp32;           // block bytes with trailers (scan input)
  uint8_t* fkeys;            // smallest / largest key of file f in slots 2f, 2f + 1
                             // of fkey_stride bytes each
  uint64_t* fkoff;           // their lengths (2 * cap_files)
  uint32_t fkey_stride;      // longest internal key the job can hold
  const uint64_t* src_koffs; // flush encoder: key offsets (n + 1)
  const uint64_t* src_voffs; // flush encoder: value offsets (n + 1)
  uint64_t* scan_scratch;    // tile sums of the prefix sums
  uint64_t cap_scan;         // capacity of the arrays scanned (for the tile sums)

  // CRC32C shift table: x^(8m) mod P for m in [0, crc_tab_n)
  const uint32_t* crc_xpow;
  uint32_t crc_xpow_n;
  const uint32_t* crc_h5;     // kCrcH5Words: the field tables of the row CRC
  const uint32_t* crc_xinv;   // kCrcXinvN: x^(-8n) mod P, back shifts by n bytes
  const uint32_t* crc_byte;   // 256: the byte table (register after byte i, from 0)
  const uint32_t* crc_ones;   // crc_xpow_n: the register after n zero bytes from all ones
  const uint32_t* crc_xpow_hi; // crc_xpow_n: x^(8 crc_xpow_n h) mod P (long shifts)
};

}  // namespace lc
