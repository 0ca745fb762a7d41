/* Test infrastructure, not product code.
 *
 * CPU restatement of the reference's compaction path, written from the
 * reference's behaviour (LevelDB 1.22 as modified by LUDA).  It is the checker
 * for the GPU engine; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  Every function names the reference code it follows.
 * Parity of this file is pinned by tests/test_oracle.py against the reference's
 * own build (oracle/_ref) and the reference's known-answer vectors
 * (util/crc32c_test.cc, util/hash_test.cc, db/dbformat_test.cc,
 * table/filter_block_test.cc).
 */
#include "lsm_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* byte buffer                                                              */

typedef struct {
  uint8_t* p;
  size_t n, cap;
} bytes;

static void b_reserve(bytes* b, size_t need) {
  if (need <= b->cap) return;
  size_t c = b->cap ? b->cap : 64;
  while (c < need) c *= 2;
  b->p = (uint8_t*)realloc(b->p, c);
  b->cap = c;
}
static void b_append(bytes* b, const void* d, size_t n) {
  b_reserve(b, b->n + n);
  if (n) memcpy(b->p + b->n, d, n);
  b->n += n;
}
static void b_putc(bytes* b, uint8_t c) { b_append(b, &c, 1); }
static void b_fixed32(bytes* b, uint32_t v) {
  uint8_t t[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
  b_append(b, t, 4);
}
static void b_fixed64(bytes* b, uint64_t v) {
  b_fixed32(b, (uint32_t)v);
  b_fixed32(b, (uint32_t)(v >> 32));
}
/* util/coding.cc:75 PutVarint32 / :95 PutVarint64: LEB128. */
static void b_varint64(bytes* b, uint64_t v) {
  while (v >= 128) {
    b_putc(b, (uint8_t)(v | 128));
    v >>= 7;
  }
  b_putc(b, (uint8_t)v);
}
static void b_free(bytes* b) {
  free(b->p);
  b->p = NULL;
  b->n = b->cap = 0;
}

static uint32_t dec32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t dec64(const uint8_t* p) { return (uint64_t)dec32(p) | ((uint64_t)dec32(p + 4) << 32); }

/* util/coding.cc:112-192 GetVarint32Ptr / GetVarint64Ptr. */
static const uint8_t* get_varint64(const uint8_t* p, const uint8_t* limit, uint64_t* v) {
  uint64_t r = 0;
  for (uint32_t shift = 0; shift <= 63 && p < limit; shift += 7) {
    uint64_t byte = *p++;
    if (byte & 128) {
      r |= (byte & 127) << shift;
    } else {
      r |= byte << shift;
      *v = r;
      return p;
    }
  }
  return NULL;
}
static const uint8_t* get_varint32(const uint8_t* p, const uint8_t* limit, uint32_t* v) {
  uint32_t r = 0;
  for (uint32_t shift = 0; shift <= 28 && p < limit; shift += 7) {
    uint32_t byte = *p++;
    if (byte & 128) {
      r |= (byte & 127) << shift;
    } else {
      r |= byte << shift;
      *v = r;
      return p;
    }
  }
  return NULL;
}

/* ------------------------------------------------------------------------ */
/* CRC32C (util/crc32c.cc:276 Extend; util/crc32c.h:29 Mask).               */
/* Castagnoli polynomial, reflected form 0x82F63B78, pre/post inversion.    */
/* Byte-at-a-time table, generated from the polynomial.                    */

static uint32_t g_crc_table[256];
__attribute__((constructor)) static void crc_init(void) {
  for (uint32_t i = 0; i < 256; i++) {
    uint32_t c = i;
    for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ 0x82F63B78u : (c >> 1);
    g_crc_table[i] = c;
  }
}
uint32_t lo_crc32c_extend(uint32_t crc, const uint8_t* data, uint64_t n) {
  uint32_t l = crc ^ 0xffffffffu;
  for (uint64_t i = 0; i < n; i++) l = g_crc_table[(l ^ data[i]) & 0xff] ^ (l >> 8);
  return l ^ 0xffffffffu;
}
uint32_t lo_crc32c_mask(uint32_t crc) { return ((crc >> 15) | (crc << 17)) + 0xa282ead8u; }

/* util/hash.cc:22-51: murmur-like hash, little-endian 4-byte words. */
uint32_t lo_hash(const uint8_t* data, uint64_t n, uint32_t seed) {
  const uint32_t m = 0xc6a4a793u;
  const uint32_t r = 24;
  const uint8_t* limit = data + n;
  uint32_t h = seed ^ (uint32_t)(n * m);
  while (data + 4 <= limit) {
    h += dec32(data);
    data += 4;
    h *= m;
    h ^= (h >> 16);
  }
  switch (limit - data) {
    case 3:
      h += (uint32_t)data[2] << 16;
      /* fall through */
    case 2:
      h += (uint32_t)data[1] << 8;
      /* fall through */
    case 1:
      h += data[0];
      h *= m;
      h ^= (h >> r);
      break;
  }
  return h;
}

/* util/bloom.cc:17-25: k = (size_t)(bits_per_key * 0.69), clamped to [1,30]. */
static size_t bloom_k(int bits_per_key) {
  size_t k = (size_t)(bits_per_key * 0.69);
  if (k < 1) k = 1;
  if (k > 30) k = 30;
  return k;
}

/* util/bloom.cc:28-54 CreateFilter: appends one filter for n keys. */
static void bloom_create(int bits_per_key, int n, const uint8_t* const* keys, const size_t* lens,
                         bytes* dst) {
  size_t bits = (size_t)n * (size_t)bits_per_key;
  if (bits < 64) bits = 64;
  size_t nbytes = (bits + 7) / 8;
  bits = nbytes * 8;
  size_t init = dst->n;
  b_reserve(dst, init + nbytes + 1);
  memset(dst->p + init, 0, nbytes);
  dst->n = init + nbytes;
  size_t k = bloom_k(bits_per_key);
  b_putc(dst, (uint8_t)k);
  uint8_t* array = dst->p + init;
  for (int i = 0; i < n; i++) {
    uint32_t h = lo_hash(keys[i], lens[i], 0xbc9f1d34u);
    const uint32_t delta = (h >> 17) | (h << 15);
    for (size_t j = 0; j < k; j++) {
      const uint32_t bitpos = (uint32_t)(h % bits);
      array[bitpos / 8] |= (uint8_t)(1u << (bitpos % 8));
      h += delta;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Internal keys (db/dbformat.h:52-65, db/dbformat.cc:51-101).              */

#define LO_MAX_SEQ ((1ull << 56) - 1)
#define LO_SEEK_TAG ((LO_MAX_SEQ << 8) | 1ull) /* PackSequenceAndType(kMax, kValueTypeForSeek) */

/* util/comparator.cc:25 Slice::compare: memcmp then length. */
static int user_cmp(const uint8_t* a, size_t al, const uint8_t* b, size_t bl) {
  size_t m = al < bl ? al : bl;
  int r = memcmp(a, b, m);
  if (r == 0) {
    if (al < bl) r = -1;
    else if (al > bl) r = 1;
  }
  return r;
}
/* db/dbformat.cc:51-67: user key ascending, then packed tag descending. */
static int icmp(const uint8_t* a, size_t al, const uint8_t* b, size_t bl) {
  int r = user_cmp(a, al - 8, b, bl - 8);
  if (r == 0) {
    uint64_t an = dec64(a + al - 8), bn = dec64(b + bl - 8);
    if (an > bn) r = -1;
    else if (an < bn) r = 1;
  }
  return r;
}

/* db/dbformat.cc:69-86 + util/comparator.cc:29-50. */
static void separator(bytes* start, const uint8_t* limit, size_t llen) {
  size_t ulen = start->n - 8;
  const uint8_t* ul = limit;
  size_t ull = llen - 8;
  bytes tmp = {0};
  b_append(&tmp, start->p, ulen);
  size_t min_len = ulen < ull ? ulen : ull;
  size_t d = 0;
  while (d < min_len && tmp.p[d] == ul[d]) d++;
  if (d < min_len) {
    uint8_t db = tmp.p[d];
    if (db < 0xff && (unsigned)db + 1 < ul[d]) {
      tmp.p[d]++;
      tmp.n = d + 1;
    }
  }
  if (tmp.n < ulen && user_cmp(start->p, ulen, tmp.p, tmp.n) < 0) {
    b_fixed64(&tmp, LO_SEEK_TAG);
    b_free(start);
    *start = tmp;
  } else {
    b_free(&tmp);
  }
}
/* db/dbformat.cc:88-101 + util/comparator.cc:52-64. */
static void successor(bytes* key) {
  size_t ulen = key->n - 8;
  bytes tmp = {0};
  b_append(&tmp, key->p, ulen);
  for (size_t i = 0; i < ulen; i++) {
    if (tmp.p[i] != 0xff) {
      tmp.p[i]++;
      tmp.n = i + 1;
      break;
    }
  }
  if (tmp.n < ulen && user_cmp(key->p, ulen, tmp.p, tmp.n) < 0) {
    b_fixed64(&tmp, LO_SEEK_TAG);
    b_free(key);
    *key = tmp;
  } else {
    b_free(&tmp);
  }
}

/* ------------------------------------------------------------------------ */
/* BlockBuilder with LUDA restart words (table/block_builder.cc:41-114):     */
/* each restart word is (offset << 8) | entries in that restart run.         */

typedef struct {
  bytes buf;
  uint32_t* restarts;
  size_t nrest, caprest;
  uint32_t counter;
  bytes last_key;
  uint32_t interval;
} blockb;

static void bb_push_restart(blockb* b, uint32_t v) {
  if (b->nrest == b->caprest) {
    b->caprest = b->caprest ? b->caprest * 2 : 16;
    b->restarts = (uint32_t*)realloc(b->restarts, b->caprest * sizeof(uint32_t));
  }
  b->restarts[b->nrest++] = v;
}
static void bb_init(blockb* b, uint32_t interval) {
  memset(b, 0, sizeof(*b));
  b->interval = interval;
  bb_push_restart(b, 0);
}
static void bb_reset(blockb* b) {
  b->buf.n = 0;
  b->nrest = 0;
  bb_push_restart(b, 0);
  b->counter = 0;
  b->last_key.n = 0;
}
static void bb_free(blockb* b) {
  b_free(&b->buf);
  b_free(&b->last_key);
  free(b->restarts);
}
static size_t bb_estimate(const blockb* b) { return b->buf.n + b->nrest * 4 + 4; }
static void bb_add(blockb* b, const uint8_t* key, size_t klen, const uint8_t* val, size_t vlen) {
  size_t shared = 0;
  if (b->counter < b->interval) {
    size_t m = b->last_key.n < klen ? b->last_key.n : klen;
    while (shared < m && b->last_key.p[shared] == key[shared]) shared++;
  } else {
    bb_push_restart(b, (uint32_t)b->buf.n);
    b->restarts[b->nrest - 2] = (b->restarts[b->nrest - 2] << 8) | b->counter;
    b->counter = 0;
  }
  size_t non_shared = klen - shared;
  b_varint64(&b->buf, shared);
  b_varint64(&b->buf, non_shared);
  b_varint64(&b->buf, vlen);
  b_append(&b->buf, key + shared, non_shared);
  b_append(&b->buf, val, vlen);
  b->last_key.n = shared;
  b_append(&b->last_key, key + shared, non_shared);
  b->counter++;
}
static void bb_finish(blockb* b) {
  if (b->nrest) b->restarts[b->nrest - 1] = (b->restarts[b->nrest - 1] << 8) | b->counter;
  for (size_t i = 0; i < b->nrest; i++) b_fixed32(&b->buf, b->restarts[i]);
  b_fixed32(&b->buf, (uint32_t)b->nrest);
}

/* ------------------------------------------------------------------------ */
/* FilterBlockBuilder (table/filter_block.cc:14-76) with the internal filter */
/* policy (db/dbformat.cc:105-115: filters hash user keys).                  */

typedef struct {
  bytes keys;
  size_t* starts;
  size_t nstarts, capstarts;
  bytes result;
  uint32_t* offsets;
  size_t noff, capoff;
  int bits_per_key;
} filterb;

static void fb_push_off(filterb* f, uint32_t v) {
  if (f->noff == f->capoff) {
    f->capoff = f->capoff ? f->capoff * 2 : 16;
    f->offsets = (uint32_t*)realloc(f->offsets, f->capoff * sizeof(uint32_t));
  }
  f->offsets[f->noff++] = v;
}
static void fb_generate(filterb* f) {
  size_t n = f->nstarts;
  if (n == 0) {
    fb_push_off(f, (uint32_t)f->result.n);
    return;
  }
  const uint8_t** ks = (const uint8_t**)malloc(n * sizeof(*ks));
  size_t* ls = (size_t*)malloc(n * sizeof(*ls));
  for (size_t i = 0; i < n; i++) {
    size_t s = f->starts[i];
    size_t e = (i + 1 < n) ? f->starts[i + 1] : f->keys.n;
    ks[i] = f->keys.p + s;
    ls[i] = (e - s) - 8; /* ExtractUserKey */
  }
  fb_push_off(f, (uint32_t)f->result.n);
  bloom_create(f->bits_per_key, (int)n, ks, ls, &f->result);
  free(ks);
  free(ls);
  f->keys.n = 0;
  f->nstarts = 0;
}
static void fb_start_block(filterb* f, uint64_t block_offset) {
  uint64_t idx = block_offset / 2048;
  while (idx > f->noff) fb_generate(f);
}
static void fb_add_key(filterb* f, const uint8_t* key, size_t len) {
  if (f->nstarts == f->capstarts) {
    f->capstarts = f->capstarts ? f->capstarts * 2 : 64;
    f->starts = (size_t*)realloc(f->starts, f->capstarts * sizeof(size_t));
  }
  f->starts[f->nstarts++] = f->keys.n;
  b_append(&f->keys, key, len);
}
static void fb_finish(filterb* f) {
  if (f->nstarts) fb_generate(f);
  uint32_t array_offset = (uint32_t)f->result.n;
  for (size_t i = 0; i < f->noff; i++) b_fixed32(&f->result, f->offsets[i]);
  b_fixed32(&f->result, array_offset);
  b_putc(&f->result, 11);
}
static void fb_free(filterb* f) {
  b_free(&f->keys);
  b_free(&f->result);
  free(f->starts);
  free(f->offsets);
}

/* ------------------------------------------------------------------------ */
/* TableBuilder (table/table_builder.cc:94-254), no compression.            */

typedef struct {
  uint32_t block_size;
  bytes out;
  uint64_t offset;
  blockb data, index;
  filterb filter;
  int has_filter;
  bytes last_key;
  int64_t num_entries;
  int pending_index;
  uint64_t pend_off, pend_size;
} tableb;

static void tb_init(tableb* t, uint32_t block_size, uint32_t restart_interval, int bits_per_key) {
  memset(t, 0, sizeof(*t));
  t->block_size = block_size;
  bb_init(&t->data, restart_interval);
  bb_init(&t->index, 1);
  t->has_filter = bits_per_key > 0;
  t->filter.bits_per_key = bits_per_key;
  if (t->has_filter) fb_start_block(&t->filter, 0);
}
static void tb_free(tableb* t) {
  b_free(&t->out);
  bb_free(&t->data);
  bb_free(&t->index);
  fb_free(&t->filter);
  b_free(&t->last_key);
}
static void handle_enc(bytes* b, uint64_t off, uint64_t size) {
  b_varint64(b, off);
  b_varint64(b, size);
}
/* WriteRawBlock (table/table_builder.cc:178-195): contents, type, masked crc. */
static void tb_write_raw(tableb* t, const uint8_t* d, size_t n, uint64_t* h_off, uint64_t* h_size) {
  *h_off = t->offset;
  *h_size = n;
  b_append(&t->out, d, n);
  uint8_t type = 0;
  uint32_t crc = lo_crc32c_extend(0, d, n);
  crc = lo_crc32c_extend(crc, &type, 1);
  b_putc(&t->out, type);
  b_fixed32(&t->out, lo_crc32c_mask(crc));
  t->offset += n + 5;
}
static void tb_write_block(tableb* t, blockb* b, uint64_t* h_off, uint64_t* h_size) {
  bb_finish(b);
  tb_write_raw(t, b->buf.p, b->buf.n, h_off, h_size);
  bb_reset(b);
}
static void tb_flush(tableb* t) {
  if (t->data.buf.n == 0) return;
  tb_write_block(t, &t->data, &t->pend_off, &t->pend_size);
  t->pending_index = 1;
  if (t->has_filter) fb_start_block(&t->filter, t->offset);
}
static void tb_add(tableb* t, const uint8_t* key, size_t klen, const uint8_t* val, size_t vlen) {
  if (t->pending_index) {
    separator(&t->last_key, key, klen);
    bytes h = {0};
    handle_enc(&h, t->pend_off, t->pend_size);
    bb_add(&t->index, t->last_key.p, t->last_key.n, h.p, h.n);
    b_free(&h);
    t->pending_index = 0;
  }
  if (t->has_filter) fb_add_key(&t->filter, key, klen);
  t->last_key.n = 0;
  b_append(&t->last_key, key, klen);
  t->num_entries++;
  bb_add(&t->data, key, klen, val, vlen);
  if (bb_estimate(&t->data) >= t->block_size) tb_flush(t);
}
static void tb_finish(tableb* t) {
  tb_flush(t);
  uint64_t f_off = 0, f_size = 0, m_off, m_size, i_off, i_size;
  if (t->has_filter) {
    fb_finish(&t->filter);
    tb_write_raw(t, t->filter.result.p, t->filter.result.n, &f_off, &f_size);
  }
  blockb meta;
  bb_init(&meta, t->data.interval);
  if (t->has_filter) {
    static const char kName[] = "filter.leveldb.BuiltinBloomFilter2";
    bytes h = {0};
    handle_enc(&h, f_off, f_size);
    bb_add(&meta, (const uint8_t*)kName, sizeof(kName) - 1, h.p, h.n);
    b_free(&h);
  }
  tb_write_block(t, &meta, &m_off, &m_size);
  bb_free(&meta);
  if (t->pending_index) {
    successor(&t->last_key);
    bytes h = {0};
    handle_enc(&h, t->pend_off, t->pend_size);
    bb_add(&t->index, t->last_key.p, t->last_key.n, h.p, h.n);
    b_free(&h);
    t->pending_index = 0;
  }
  tb_write_block(t, &t->index, &i_off, &i_size);
  /* Footer::EncodeTo (table/format.cc:31-40). */
  bytes f = {0};
  handle_enc(&f, m_off, m_size);
  handle_enc(&f, i_off, i_size);
  b_reserve(&f, 40);
  while (f.n < 40) b_putc(&f, 0);
  b_fixed32(&f, 0x8b80fb57u);
  b_fixed32(&f, 0xdb477524u);
  b_append(&t->out, f.p, f.n);
  t->offset += f.n;
  b_free(&f);
}

/* ------------------------------------------------------------------------ */
/* Table decoding (table/format.cc:42 Footer::DecodeFrom, table/block.cc     */
/* :170 DecodeEntry, :340 ParseNextKey).                                     */

typedef struct {
  uint64_t koff; /* into entry key store */
  uint32_t klen;
  const uint8_t* val;
  uint32_t vlen;
} lo_entry;

typedef struct {
  lo_entry* e;
  size_t n, cap;
  bytes keys;
} entry_list;

static void el_push(entry_list* l, const uint8_t* key, uint32_t klen, const uint8_t* val,
                    uint32_t vlen) {
  if (l->n == l->cap) {
    l->cap = l->cap ? l->cap * 2 : 1024;
    l->e = (lo_entry*)realloc(l->e, l->cap * sizeof(lo_entry));
  }
  l->e[l->n].koff = l->keys.n;
  l->e[l->n].klen = klen;
  l->e[l->n].val = val;
  l->e[l->n].vlen = vlen;
  l->n++;
  b_append(&l->keys, key, klen);
}

/* Decodes every entry of one block; returns 0 on success. */
static int decode_block(const uint8_t* d, uint64_t n, entry_list* out) {
  if (n < 4) return -1;
  uint32_t nr = dec32(d + n - 4);
  if ((uint64_t)nr > (n - 4) / 4) return -1;
  uint64_t limit = n - 4 - 4ull * nr;
  const uint8_t* p = d;
  const uint8_t* lim = d + limit;
  bytes key = {0};
  while (p < lim) {
    uint32_t shared, non_shared, vlen;
    if ((p = get_varint32(p, lim, &shared)) == NULL) goto bad;
    if ((p = get_varint32(p, lim, &non_shared)) == NULL) goto bad;
    if ((p = get_varint32(p, lim, &vlen)) == NULL) goto bad;
    if ((uint64_t)(lim - p) < (uint64_t)non_shared + vlen) goto bad;
    if (key.n < shared) goto bad;
    key.n = shared;
    b_append(&key, p, non_shared);
    p += non_shared;
    el_push(out, key.p, (uint32_t)key.n, p, vlen);
    p += vlen;
  }
  b_free(&key);
  return 0;
bad:
  b_free(&key);
  return -1;
}

static int decode_table(const uint8_t* d, uint64_t n, entry_list* out) {
  if (n < 48) return -1;
  const uint8_t* foot = d + n - 48;
  if (dec32(foot + 40) != 0x8b80fb57u || dec32(foot + 44) != 0xdb477524u) return -1;
  uint64_t m_off, m_size, i_off, i_size;
  const uint8_t* p = foot;
  if ((p = get_varint64(p, foot + 40, &m_off)) == NULL) return -1;
  if ((p = get_varint64(p, foot + 40, &m_size)) == NULL) return -1;
  if ((p = get_varint64(p, foot + 40, &i_off)) == NULL) return -1;
  if ((p = get_varint64(p, foot + 40, &i_size)) == NULL) return -1;
  if (i_off > n || i_size + 5 > n - i_off) return -1;
  entry_list idx = {0};
  if (decode_block(d + i_off, i_size, &idx) != 0) goto bad;
  for (size_t i = 0; i < idx.n; i++) {
    const uint8_t* v = idx.e[i].val;
    uint64_t b_off, b_size;
    const uint8_t* q = v;
    if ((q = get_varint64(q, v + idx.e[i].vlen, &b_off)) == NULL) goto bad;
    if ((q = get_varint64(q, v + idx.e[i].vlen, &b_size)) == NULL) goto bad;
    if (b_off > n || b_size + 5 > n - b_off) goto bad;
    if (decode_block(d + b_off, b_size, out) != 0) goto bad;
  }
  free(idx.e);
  b_free(&idx.keys);
  return 0;
bad:
  free(idx.e);
  b_free(&idx.keys);
  return -1;
}

/* ------------------------------------------------------------------------ */
/* Compaction.                                                              */

typedef struct {
  bytes data;
  bytes smallest, largest;
  uint64_t entries;
} lo_file;

struct lo_result {
  lo_file* files;
  int n, cap;
};

struct lo_buf {
  bytes b;
};

static void res_push(lo_result* r, tableb* t, const bytes* smallest, const bytes* largest) {
  if (r->n == r->cap) {
    r->cap = r->cap ? r->cap * 2 : 8;
    r->files = (lo_file*)realloc(r->files, r->cap * sizeof(lo_file));
  }
  lo_file* f = &r->files[r->n++];
  memset(f, 0, sizeof(*f));
  f->data = t->out; /* take ownership */
  t->out.p = NULL;
  t->out.n = t->out.cap = 0;
  b_append(&f->smallest, smallest->p, smallest->n);
  b_append(&f->largest, largest->p, largest->n);
  f->entries = (uint64_t)t->num_entries;
}

/* Compaction::IsBaseLevelForKey (db/version_set.cc:1535-1554), one pointer
 * per level advanced monotonically as in the reference. */
static int is_base_level(const lo_job* job, size_t* ptrs, const uint8_t* ukey, size_t ulen) {
  for (int lvl = job->level + 2; lvl < 7; lvl++) {
    /* files of this level occupy a contiguous slice of base_files */
    size_t begin = 0, end = 0;
    int found = 0;
    for (int i = 0; i < job->n_base_files; i++) {
      if (job->base_files[i].level == lvl) {
        if (!found) begin = (size_t)i;
        found = 1;
        end = (size_t)i + 1;
      }
    }
    if (!found) continue;
    size_t nfiles = end - begin;
    for (; ptrs[lvl] < nfiles;) {
      const lo_file_range* f = &job->base_files[begin + ptrs[lvl]];
      if (user_cmp(ukey, ulen, f->largest, f->largest_len - 8) <= 0) {
        if (user_cmp(ukey, ulen, f->smallest, f->smallest_len - 8) >= 0) return 0;
        break;
      }
      ptrs[lvl]++;
    }
  }
  return 1;
}

lo_result* lo_compact(const lo_job* job, int* status) {
  *status = 0;
  lo_result* res = (lo_result*)calloc(1, sizeof(lo_result));
  if (job->n_runs <= 0 || job->restart_interval < 1) {
    *status = 1;
    return res;
  }
  int nr = job->n_runs;
  entry_list* runs = (entry_list*)calloc((size_t)nr, sizeof(entry_list));
  int ti = 0;
  for (int r = 0; r < nr; r++) {
    for (int k = 0; k < job->run_table_count[r]; k++, ti++) {
      if (ti >= job->n_tables ||
          decode_table(job->tables[ti].data, job->tables[ti].size, &runs[r]) != 0) {
        *status = 2;
        goto done;
      }
    }
    for (size_t i = 0; i < runs[r].n; i++)
      if (runs[r].e[i].klen < 8) {
        *status = 2;
        goto done;
      }
  }

  {
    size_t* cur = (size_t*)calloc((size_t)nr, sizeof(size_t));
    size_t level_ptrs[7] = {0};
    const int64_t max_overlap = 10 * (int64_t)job->max_file_size; /* db/version_set.cc:31 */
    size_t gp_index = 0;
    int seen_key = 0;
    int64_t overlapped = 0;
    bytes cur_user = {0};
    int has_cur_user = 0;
    uint64_t last_seq = LO_MAX_SEQ;
    tableb tb;
    int open = 0;
    bytes smallest = {0}, largest = {0};

    for (;;) {
      /* MergingIterator::FindSmallest (table/merger.cc:148): first child
       * with the smallest key wins ties. */
      int best = -1;
      for (int r = 0; r < nr; r++) {
        if (cur[r] >= runs[r].n) continue;
        if (best < 0) {
          best = r;
          continue;
        }
        const lo_entry* a = &runs[r].e[cur[r]];
        const lo_entry* b = &runs[best].e[cur[best]];
        if (icmp(runs[r].keys.p + a->koff, a->klen, runs[best].keys.p + b->koff, b->klen) < 0)
          best = r;
      }
      if (best < 0) break;
      const lo_entry* e = &runs[best].e[cur[best]];
      const uint8_t* key = runs[best].keys.p + e->koff;
      size_t klen = e->klen;
      cur[best]++;

      /* Compaction::ShouldStopBefore (db/version_set.cc:1556-1579). */
      while (gp_index < (size_t)job->n_grandparents &&
             icmp(key, klen, job->grandparents[gp_index].largest,
                  job->grandparents[gp_index].largest_len) > 0) {
        if (seen_key) overlapped += (int64_t)job->grandparents[gp_index].file_size;
        gp_index++;
      }
      seen_key = 1;
      int stop = 0;
      if (overlapped > max_overlap) {
        overlapped = 0;
        stop = 1;
      }
      if (stop && open) {
        tb_finish(&tb);
        res_push(res, &tb, &smallest, &largest);
        tb_free(&tb);
        open = 0;
      }

      /* Drop rule (db/db_impl.cc:1113-1147). */
      int drop = 0;
      uint64_t tag = dec64(key + klen - 8);
      uint8_t type = (uint8_t)(tag & 0xff);
      uint64_t seq = tag >> 8;
      if (type > 1) { /* ParseInternalKey fails: keep and reset */
        cur_user.n = 0;
        has_cur_user = 0;
        last_seq = LO_MAX_SEQ;
      } else {
        if (!has_cur_user || user_cmp(key, klen - 8, cur_user.p, cur_user.n) != 0) {
          cur_user.n = 0;
          b_append(&cur_user, key, klen - 8);
          has_cur_user = 1;
          last_seq = LO_MAX_SEQ;
        }
        if (last_seq <= job->smallest_snapshot) {
          drop = 1;
        } else if (type == 0 && seq <= job->smallest_snapshot &&
                   is_base_level(job, level_ptrs, key, klen - 8)) {
          drop = 1;
        }
        last_seq = seq;
      }

      if (!drop) {
        if (!open) {
          tb_init(&tb, job->block_size, job->restart_interval, job->bits_per_key);
          open = 1;
        }
        if (tb.num_entries == 0) {
          smallest.n = 0;
          b_append(&smallest, key, klen);
        }
        largest.n = 0;
        b_append(&largest, key, klen);
        tb_add(&tb, key, klen, e->val, e->vlen);
        if (tb.offset >= job->max_file_size) {
          tb_finish(&tb);
          res_push(res, &tb, &smallest, &largest);
          tb_free(&tb);
          open = 0;
        }
      }
    }
    if (open) {
      tb_finish(&tb);
      res_push(res, &tb, &smallest, &largest);
      tb_free(&tb);
    }
    free(cur);
    b_free(&cur_user);
    b_free(&smallest);
    b_free(&largest);
  }
done:
  for (int r = 0; r < nr; r++) {
    free(runs[r].e);
    b_free(&runs[r].keys);
  }
  free(runs);
  return res;
}

int lo_result_nfiles(const lo_result* r) { return r->n; }
const uint8_t* lo_result_file(const lo_result* r, int i, uint64_t* len) {
  *len = r->files[i].data.n;
  return r->files[i].data.p;
}
const uint8_t* lo_result_smallest(const lo_result* r, int i, uint32_t* len) {
  *len = (uint32_t)r->files[i].smallest.n;
  return r->files[i].smallest.p;
}
const uint8_t* lo_result_largest(const lo_result* r, int i, uint32_t* len) {
  *len = (uint32_t)r->files[i].largest.n;
  return r->files[i].largest.p;
}
uint64_t lo_result_entries(const lo_result* r, int i) { return r->files[i].entries; }
void lo_result_free(lo_result* r) {
  for (int i = 0; i < r->n; i++) {
    b_free(&r->files[i].data);
    b_free(&r->files[i].smallest);
    b_free(&r->files[i].largest);
  }
  free(r->files);
  free(r);
}

lo_buf* lo_build_table(uint32_t block_size, uint32_t restart_interval, int bits_per_key,
                       int64_t n, const uint8_t* keys, const uint64_t* key_offs,
                       const uint8_t* vals, const uint64_t* val_offs) {
  tableb tb;
  tb_init(&tb, block_size, restart_interval, bits_per_key);
  for (int64_t i = 0; i < n; i++)
    tb_add(&tb, keys + key_offs[i], key_offs[i + 1] - key_offs[i], vals + val_offs[i],
           val_offs[i + 1] - val_offs[i]);
  tb_finish(&tb);
  lo_buf* b = (lo_buf*)calloc(1, sizeof(lo_buf));
  b->b = tb.out;
  tb.out.p = NULL;
  tb_free(&tb);
  return b;
}

lo_buf* lo_read_table(const uint8_t* data, uint64_t size, int* status) {
  entry_list l = {0};
  lo_buf* b = (lo_buf*)calloc(1, sizeof(lo_buf));
  *status = decode_table(data, size, &l);
  if (*status == 0) {
    for (size_t i = 0; i < l.n; i++) {
      b_fixed32(&b->b, l.e[i].klen);
      b_append(&b->b, l.keys.p + l.e[i].koff, l.e[i].klen);
      b_fixed32(&b->b, l.e[i].vlen);
      b_append(&b->b, l.e[i].val, l.e[i].vlen);
    }
  }
  free(l.e);
  b_free(&l.keys);
  return b;
}

const uint8_t* lo_buf_data(const lo_buf* b, uint64_t* len) {
  *len = b->b.n;
  return b->b.p;
}
void lo_buf_free(lo_buf* b) {
  b_free(&b->b);
  free(b);
}

lo_buf* lo_bloom(int bits_per_key, int n, const uint8_t* keys, const uint64_t* key_offs) {
  lo_buf* b = (lo_buf*)calloc(1, sizeof(lo_buf));
  const uint8_t** ks = (const uint8_t**)malloc((size_t)(n ? n : 1) * sizeof(*ks));
  size_t* ls = (size_t*)malloc((size_t)(n ? n : 1) * sizeof(*ls));
  for (int i = 0; i < n; i++) {
    ks[i] = keys + key_offs[i];
    ls[i] = key_offs[i + 1] - key_offs[i];
  }
  bloom_create(bits_per_key, n, ks, ls, &b->b);
  free(ks);
  free(ls);
  return b;
}

lo_buf* lo_separator(const uint8_t* a, uint32_t alen, const uint8_t* bb, uint32_t blen) {
  lo_buf* r = (lo_buf*)calloc(1, sizeof(lo_buf));
  b_append(&r->b, a, alen);
  separator(&r->b, bb, blen);
  return r;
}
lo_buf* lo_successor(const uint8_t* a, uint32_t alen) {
  lo_buf* r = (lo_buf*)calloc(1, sizeof(lo_buf));
  b_append(&r->b, a, alen);
  successor(&r->b);
  return r;
}
