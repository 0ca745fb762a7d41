"""Seeded synthetic compaction workloads.

The reference publishes no dataset for this path; every input is synthetic,
drawn from a seeded ``numpy.random.Generator`` (PCG64) with the shapes and
value distributions the workload names:

* ``plain_l0_l1``   2 overlapping L0 + 2 L1 tables, ~20k entries each,
                    ``%016d`` keys (db/db_bench.cc:729) of uniform ints in
                    [0, 2^20), 100-byte values, ~10% of keys rewritten by newer
                    tables, 2% deletion markers, no snapshots.
* ``l1_l2_at_size`` 1 L1 table of 2 MiB over 32 L2 tables of 2 MiB; Zipf(0.99)
                    ids over 2^24; user keys 8-64 bytes (uniform per id) with
                    shared prefixes; lognormal values (median 128 B, sigma 1.0,
                    clipped to [0, 4096]); 5% deletion markers; snapshots at the
                    0.25/0.5/0.75 sequence quantiles; L3 files covering the lower
                    half of the key range (the upper half is bottommost).
* ``batched_job``   one of the 64 jobs of the batched workload: input size
                    log-uniform in [1, 64] MiB, 2-12 tables, 16-byte keys and
                    100-byte values.
* ``large_l2_l3``   1 + 15 tables of 64 MiB; run "A" 8-byte big-endian uniform
                    u64 keys with 1 KiB values, run "B" 24-byte keys with 32-byte
                    values; 64 MiB output files, 1 snapshot, 1% deletion markers.

Every generator takes ``scale`` to shrink table sizes for quick parity tests;
``scale=1`` is the full size.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .job import CompactionJob, Entries, FileMeta, TableOptions

TYPE_DELETION = 0  # kTypeDeletion (db/dbformat.h:52)
TYPE_VALUE = 1  # kTypeValue


def _pack_entries(ukeys: List[bytes], seqs: np.ndarray, types: np.ndarray,
                  vlens: np.ndarray, rng: np.random.Generator) -> Entries:
    """Internal keys from user keys + tags; values are random bytes."""
    n = len(ukeys)
    tags = (seqs.astype(np.uint64) << np.uint64(8)) | types.astype(np.uint64)
    tag_bytes = tags.astype("<u8").tobytes()
    klens = np.fromiter((len(k) + 8 for k in ukeys), np.uint64, n)
    koffs = np.zeros(n + 1, np.uint64)
    koffs[1:] = np.cumsum(klens)
    kb = bytearray(int(koffs[-1]))
    pos = 0
    for i, k in enumerate(ukeys):
        kb[pos:pos + len(k)] = k
        pos += len(k)
        kb[pos:pos + 8] = tag_bytes[8 * i:8 * i + 8]
        pos += 8
    vlens = np.where(types == TYPE_DELETION, 0, vlens).astype(np.uint64)
    voffs = np.zeros(n + 1, np.uint64)
    voffs[1:] = np.cumsum(vlens)
    vals = rng.integers(0, 256, int(voffs[-1]), dtype=np.uint8)
    return Entries(np.frombuffer(bytes(kb), np.uint8).copy(), koffs, vals, voffs)


def _pack_fixed(ukeys: np.ndarray, seqs: np.ndarray, types: np.ndarray, vlens: np.ndarray,
                rng: np.random.Generator) -> Entries:
    """Vectorised ``_pack_entries`` for fixed-width user keys ``(n, L)`` uint8."""
    n, L = ukeys.shape
    tags = ((seqs.astype(np.uint64) << np.uint64(8)) | types.astype(np.uint64)).astype("<u8")
    ik = np.empty((n, L + 8), np.uint8)
    ik[:, :L] = ukeys
    ik[:, L:] = tags.view(np.uint8).reshape(n, 8)
    koffs = (np.arange(n + 1, dtype=np.uint64) * np.uint64(L + 8))
    vlens = np.where(types == TYPE_DELETION, 0, vlens).astype(np.uint64)
    voffs = np.zeros(n + 1, np.uint64)
    voffs[1:] = np.cumsum(vlens)
    vals = rng.integers(0, 256, int(voffs[-1]), dtype=np.uint8)
    return Entries(ik.reshape(-1), koffs, vals, voffs)


def _decimal16(ids: np.ndarray) -> np.ndarray:
    """``snprintf("%016d")`` of non-negative ints as an (n, 16) uint8 array."""
    out = np.empty((len(ids), 16), np.uint8)
    v = ids.astype(np.int64).copy()
    for c in range(15, -1, -1):
        out[:, c] = 48 + (v % 10)
        v //= 10
    return out


def _file(level: int, number: int, e: Entries) -> FileMeta:
    return FileMeta(level=level, number=number, smallest=e.key(0), largest=e.key(e.n - 1),
                    entries=e)


def _split_sorted(order_keys: np.ndarray, nparts: int) -> List[np.ndarray]:
    return [p for p in np.array_split(np.arange(len(order_keys)), nparts) if len(p)]


def _unique_fill(rng, have: set, count: int, draw) -> np.ndarray:
    out = []
    seen = set()
    while len(out) < count:
        for x in draw(count - len(out) + 16).tolist():
            if x not in seen and x not in have:
                seen.add(x)
                out.append(x)
                if len(out) == count:
                    break
    return np.array(out, np.int64)


def l0_l1_job(seed: int, n0: int, n1: int, entries_per_table: int, key_space: int = 1 << 20,
              rewrite_frac: float = 0.10, tomb_frac: float = 0.02, value_len: int = 100,
              options: TableOptions = None, name: str = "l0_l1") -> CompactionJob:
    """A level-0 job: ``n0`` overlapping L0 tables over ``n1`` L1 tables."""
    rng = np.random.default_rng(seed)
    options = options or TableOptions()
    files: List[FileMeta] = []
    number = 1
    seq = 1
    # L1: n1 * entries unique keys, oldest sequence numbers, split by key range.
    n_l1 = n1 * entries_per_table
    l1_ids = np.sort(rng.choice(key_space, size=n_l1, replace=False)) if n_l1 else np.zeros(0, np.int64)
    prior = set(l1_ids.tolist())
    if n_l1:
        seqs = seq + rng.permutation(n_l1)
        seq += n_l1
        types = np.where(rng.random(n_l1) < tomb_frac, TYPE_DELETION, TYPE_VALUE)
        e = _pack_fixed(_decimal16(l1_ids), seqs, types, np.full(n_l1, value_len), rng)
        for part in _split_sorted(l1_ids, n1):
            files.append(_file(1, number, e.slice(int(part[0]), int(part[-1]) + 1)))
            number += 1
    # L0 tables, each newer than everything before it.
    for _ in range(n0):
        n = entries_per_table
        n_rw = int(round(rewrite_frac * n)) if prior else 0
        rw = rng.choice(np.array(sorted(prior), np.int64), size=min(n_rw, len(prior)),
                        replace=False) if n_rw else np.zeros(0, np.int64)
        fresh = _unique_fill(rng, set(rw.tolist()), n - len(rw),
                             lambda m: rng.integers(0, key_space, m))
        ids = np.sort(np.concatenate([rw, fresh]))
        seqs = seq + rng.permutation(n)
        seq += n
        types = np.where(rng.random(n) < tomb_frac, TYPE_DELETION, TYPE_VALUE)
        e = _pack_fixed(_decimal16(ids), seqs, types, np.full(n, value_len), rng)
        files.append(_file(0, number, e))
        number += 1
        prior.update(ids.tolist())
    return CompactionJob(level=0, files=files, snapshots=[], last_sequence=seq - 1,
                         options=options, name=name)


def plain_l0_l1(seed: int = 0, scale: float = 1.0) -> CompactionJob:
    """2 overlapping L0 + 2 L1 tables of ~20k entries (the CPU-runnable case)."""
    n = max(8, int(20000 * scale))
    return l0_l1_job(seed, n0=2, n1=2, entries_per_table=n, name="plain_l0_l1")


def batched_job(seed: int, scale: float = 1.0) -> CompactionJob:
    """One job of the 64-job batched workload."""
    rng = np.random.default_rng(10_000 + seed)
    size_mib = math.exp(rng.uniform(math.log(1.0), math.log(64.0))) * scale
    n_tables = int(rng.integers(2, 13))
    n0 = int(rng.integers(1, min(4, n_tables - 1) + 1))
    n1 = n_tables - n0
    per_table = max(8, int(size_mib * (1 << 20) / n_tables / 130))
    return l0_l1_job(20_000 + seed, n0=n0, n1=n1, entries_per_table=per_table,
                     key_space=1 << 26, name=f"batched_{seed}")


# --------------------------------------------------------------------------
# L1 -> L2 at size


def _splitmix64(x: np.ndarray) -> np.ndarray:
    z = (x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15))
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def zipf_ids(rng: np.random.Generator, n: int, s: float = 0.99, space: int = 1 << 24) -> np.ndarray:
    """Zipf(s) ranks over [1, space] by inverting the continuous CDF
    ``(k^(1-s) - 1) / (space^(1-s) - 1)``; ranks are scattered over the id
    space by an odd multiplier (a bijection mod 2^24)."""
    u = rng.random(n)
    a = 1.0 - s
    k = np.floor((1.0 + u * (space ** a - 1.0)) ** (1.0 / a)).astype(np.int64)
    k = np.clip(k, 1, space) - 1
    return (k * 0x9E3779B1) % space


def varlen_user_key(ids: np.ndarray) -> List[bytes]:
    """8-64 byte keys, length uniform per id; most share one of 32 prefixes."""
    h = _splitmix64(ids)
    h2 = _splitmix64(h)
    lens = 8 + (h % np.uint64(57)).astype(np.int64)
    grps = ((h >> np.uint64(8)) % np.uint64(32)).astype(np.int64)
    out = []
    for i in range(len(ids)):
        fill = ("%016x" % int(h2[i])) * 4
        hexid = "%08x" % int(ids[i])
        L = int(lens[i])
        if L >= 12:
            k = ("t%02d:" % int(grps[i])) + hexid + fill[:L - 12]
        else:
            k = hexid + fill[:L - 8]
        out.append(k.encode())
    return out


def _lognormal_lens(rng, n, median=128.0, sigma=1.0, lo=0, hi=4096):
    return np.clip(np.round(rng.lognormal(math.log(median), sigma, n)), lo, hi).astype(np.int64)


def l1_l2_at_size(seed: int = 1, scale: float = 1.0, n_l2_tables: int = 32,
                  n_l3_files: int = 160) -> CompactionJob:
    rng = np.random.default_rng(seed)
    table_bytes = int((2 << 20) * scale)
    est_entry = 44 + 205 + 4  # mean internal key + mean clipped value + header
    n_l2 = max(16, n_l2_tables * table_bytes // est_entry)
    n_l1 = max(8, table_bytes // est_entry)
    # L2 ids: distinct Zipf draws in draw order; ~3% get a second version.
    l2_ids = _unique_fill(rng, set(), n_l2, lambda m: zipf_ids(rng, 4 * m))
    l1_ids = _unique_fill(rng, set(), n_l1, lambda m: zipf_ids(rng, 4 * m))
    dup = l2_ids[rng.random(len(l2_ids)) < 0.03]
    # Records in age order per key: L2 version(s) first, then the L1 version.
    rec_ids = np.concatenate([l2_ids, dup, l1_ids]).astype(np.int64)
    n_l2_recs = len(l2_ids) + len(dup)
    n_total = len(rec_ids)
    seqs = 1 + rng.permutation(n_total)
    # A key's newer record must hold the larger sequence number: sort the
    # sequence numbers drawn for each key's records and hand them out in age
    # order.
    order = np.lexsort((np.arange(n_total), rec_ids))
    sorted_ids = rec_ids[order]
    starts = np.flatnonzero(np.r_[True, sorted_ids[1:] != sorted_ids[:-1]])
    ends = np.r_[starts[1:], n_total]
    multi = np.flatnonzero(ends - starts > 1)
    for g in multi:
        idx = order[starts[g]:ends[g]]
        seqs[idx] = np.sort(seqs[idx])
    l2_seq = seqs[:n_l2_recs]
    l1_seq = seqs[n_l2_recs:]
    recs_l2 = [(int(i), 0) for i in l2_ids] + [(int(i), 1) for i in dup]

    def level_entries(ids_list, seq_list):
        ukeys = varlen_user_key(np.array(ids_list, np.int64))
        order = sorted(range(len(ukeys)), key=lambda j: (ukeys[j], -int(seq_list[j])))
        uk = [ukeys[j] for j in order]
        sq = np.array([seq_list[j] for j in order], np.int64)
        n = len(uk)
        types = np.where(rng.random(n) < 0.05, TYPE_DELETION, TYPE_VALUE)
        return _pack_entries(uk, sq, types, _lognormal_lens(rng, n), rng), uk

    e2, uk2 = level_entries([r[0] for r in recs_l2], l2_seq)
    e1, uk1 = level_entries(list(l1_ids), l1_seq)
    files: List[FileMeta] = []
    number = 1
    files.append(_file(1, number, e1))
    number += 1
    # split L2 into tables of ~table_bytes, never between versions of one key
    sizes = (np.diff(e2.koffs) + np.diff(e2.voffs) + 3).astype(np.int64)
    cum = np.cumsum(sizes)
    cuts = [0]
    target = table_bytes
    for j in range(1, e2.n):
        if cum[j - 1] >= target and uk2[j] != uk2[j - 1]:
            cuts.append(j)
            target = cum[j - 1] + table_bytes
    cuts.append(e2.n)
    for a, b in zip(cuts[:-1], cuts[1:]):
        files.append(_file(2, number, e2.slice(a, b)))
        number += 1
    # L3: files over the lower half of the key range, metadata only.
    all_keys = sorted(set(uk1) | set(uk2))
    half = all_keys[:len(all_keys) // 2]
    if len(half) >= 2 * n_l3_files:
        idx = np.linspace(0, len(half) - 1, 2 * n_l3_files).astype(np.int64)
        for f in range(n_l3_files):
            lo_k, hi_k = half[idx[2 * f]], half[idx[2 * f + 1]]
            files.append(FileMeta(level=3, number=number,
                                  smallest=lo_k + (1 << 8 | 1).to_bytes(8, "little"),
                                  largest=hi_k + (1 << 8 | 1).to_bytes(8, "little"),
                                  file_size=2 << 20))
            number += 1
    last = int(n_total)
    snaps = sorted({max(1, int(q * last)) for q in (0.25, 0.5, 0.75)})
    return CompactionJob(level=1, files=files, snapshots=snaps, last_sequence=last,
                         options=TableOptions(), name="l1_l2_at_size")


# --------------------------------------------------------------------------
# large L2 -> L3


def large_l2_l3(run: str = "A", seed: int = 4, scale: float = 1.0,
                n_l3_tables: int = 15) -> CompactionJob:
    rng = np.random.default_rng(seed + (0 if run == "A" else 100))
    table_bytes = int((64 << 20) * scale)
    if run == "A":
        klen, vlen = 8, 1024
    else:
        klen, vlen = 24, 32
    per_table = max(8, table_bytes // (klen + 8 + vlen + 3))
    n3 = per_table * n_l3_tables
    n2 = per_table
    ids3 = np.unique(rng.integers(0, 2 ** 63, n3, dtype=np.int64).astype(np.uint64))
    n_rw = n2 // 10
    rw = rng.choice(ids3, size=min(n_rw, len(ids3)), replace=False)
    fresh = rng.integers(0, 2 ** 63, n2 - len(rw), dtype=np.int64).astype(np.uint64)
    ids2 = np.unique(np.concatenate([rw, fresh]))
    n_total = len(ids3) + len(ids2)
    seqs = 1 + rng.permutation(n_total)
    s3 = seqs[:len(ids3)].copy()
    s2 = seqs[len(ids3):].copy()
    # shared keys: the L2 version is the newer one
    common, i3, i2 = np.intersect1d(ids3, ids2, return_indices=True)
    hi = np.maximum(s3[i3], s2[i2])
    lo = np.minimum(s3[i3], s2[i2])
    s2[i2], s3[i3] = hi, lo

    def keys_of(ids):
        be = ids.astype(">u8").view(np.uint8).reshape(-1, 8)
        if klen == 8:
            return be
        ext = _splitmix64(ids)
        ext2 = _splitmix64(ext)
        tail = np.concatenate([ext.astype(">u8").view(np.uint8).reshape(-1, 8),
                               ext2.astype(">u8").view(np.uint8).reshape(-1, 8)], axis=1)
        return np.concatenate([be, tail], axis=1)

    def entries(ids, sq):
        n = len(ids)
        types = np.where(rng.random(n) < 0.01, TYPE_DELETION, TYPE_VALUE)
        return _pack_fixed(keys_of(ids), sq, types, np.full(n, vlen), rng)

    e2 = entries(ids2, s2)
    e3 = entries(ids3, s3)
    opts = TableOptions(max_file_size=int((64 << 20) * scale) if scale < 1 else 64 << 20)
    opts.max_file_size = max(opts.max_file_size, 1 << 20)
    files = [_file(2, 1, e2)]
    number = 2
    for part in np.array_split(np.arange(e3.n), n_l3_tables):
        if len(part):
            files.append(_file(3, number, e3.slice(int(part[0]), int(part[-1]) + 1)))
            number += 1
    last = int(n_total)
    return CompactionJob(level=2, files=files, snapshots=[last // 2], last_sequence=last,
                         options=opts, name=f"large_l2_l3_{run}")
