"""Small compaction jobs that exercise the edge cases the reference's own
tests and code paths cover: single entries, everything dropped, restart
intervals 1/2/16, block sizes at the clamp limits, no filter policy,
unparseable internal keys, 0xff user keys (FindShortSuccessor), long shared
prefixes (FindShortestSeparator), snapshots between versions, identical
internal keys in two merge children, empty values, many output files and
grandparent cuts.  Every job is seeded and deterministic.
"""
from __future__ import annotations

import numpy as np

from luda_b200.job import CompactionJob, Entries, FileMeta, TableOptions, internal_key
from luda_b200 import workloads


def _table(level, number, items):
    """items: list of (user_key, seq, type, value), sorted here."""
    items = sorted(items, key=lambda t: (t[0], -t[1]))
    keys = [internal_key(u, s, t) for (u, s, t, v) in items]
    vals = [v for (u, s, t, v) in items]
    e = Entries.from_lists(keys, vals)
    return FileMeta(level=level, number=number, smallest=keys[0], largest=keys[-1], entries=e)


def single_entry():
    return CompactionJob(level=0, files=[_table(0, 1, [(b"key00001", 5, 1, b"v")])],
                         snapshots=[], last_sequence=5, name="single_entry")


def all_dropped():
    # tombstones over older values at the bottommost level: nothing survives
    l0 = _table(0, 2, [(b"k%07d" % i, 100 + i, 0, b"") for i in range(50)])
    l1 = _table(1, 1, [(b"k%07d" % i, 1 + i, 1, b"x" * 20) for i in range(50)])
    return CompactionJob(level=0, files=[l0, l1], snapshots=[], last_sequence=200,
                         name="all_dropped")


def options_variant(restart_interval=16, block_size=4096, bits_per_key=10, seed=7, n=3000,
                    max_file_size=2 << 20, name=None):
    opts = TableOptions(block_size=block_size, restart_interval=restart_interval,
                        bits_per_key=bits_per_key, max_file_size=max_file_size)
    job = workloads.l0_l1_job(seed, n0=2, n1=2, entries_per_table=n, options=opts,
                              name=name or f"opts_r{restart_interval}_b{block_size}_f{bits_per_key}")
    return job


def unparseable_keys():
    rng = np.random.default_rng(11)
    items0 = []
    for i in range(400):
        t = 1 if i % 37 else 2  # type byte 2: ParseInternalKey fails
        items0.append((b"u%06d" % (2 * i), 1000 + i, t, rng.bytes(30)))
    items1 = [(b"u%06d" % (2 * i), 10 + i, 1, rng.bytes(30)) for i in range(400)]
    return CompactionJob(level=0, files=[_table(0, 2, items0), _table(1, 1, items1)],
                         snapshots=[], last_sequence=5000, name="unparseable_keys")


def ff_keys_and_prefixes():
    rng = np.random.default_rng(12)
    items = []
    seq = 1
    for i in range(600):
        if i % 3 == 0:
            u = b"\xff" * (1 + i % 5) + bytes([i % 251])
        elif i % 3 == 1:
            u = b"shared/prefix/that/is/long/" + b"%05d" % i + b"\xfe\xff"
        else:
            u = bytes(rng.integers(0, 256, 1 + i % 40, dtype=np.uint8))
        items.append((u, seq, 1, rng.bytes(int(rng.integers(0, 300)))))
        seq += 1
    # dedupe user keys within the table
    seen, uniq = set(), []
    for it in items:
        if it[0] not in seen:
            seen.add(it[0])
            uniq.append(it)
    opts = TableOptions(block_size=1024)
    return CompactionJob(level=0, files=[_table(0, 1, uniq)], snapshots=[], last_sequence=seq,
                         options=opts, name="ff_keys_and_prefixes")


def snapshot_versions():
    rng = np.random.default_rng(13)
    l1, l0 = [], []
    for i in range(2000):
        u = b"sv%06d" % i
        l1.append((u, 1 + i, 1, rng.bytes(40)))
        if i % 2 == 0:
            l0.append((u, 3000 + i, 1 if i % 10 else 0, rng.bytes(40) if i % 10 else b""))
    # a second newer version of some keys in another L0 table
    l0b = [(b"sv%06d" % i, 6000 + i, 1, rng.bytes(40)) for i in range(0, 2000, 7)]
    snaps = [2500, 4000, 5500]
    return CompactionJob(level=0, files=[_table(1, 1, l1), _table(0, 2, l0), _table(0, 3, l0b)],
                         snapshots=snaps, last_sequence=9000, name="snapshot_versions")


def identical_internal_keys():
    # the same internal key in two level-0 tables: the first merge child wins
    a = [(b"dup%05d" % i, 100 + i, 1, b"A" * 10) for i in range(300)]
    b = [(b"dup%05d" % i, 100 + i, 1, b"B" * 12) for i in range(0, 300, 3)]
    return CompactionJob(level=0, files=[_table(0, 1, a), _table(0, 2, b)], snapshots=[50],
                         last_sequence=1000, name="identical_internal_keys")


def empty_values():
    items = [(b"e%08d" % i, 1 + i, 1, b"") for i in range(5000)]
    return CompactionJob(level=0, files=[_table(0, 1, items)], snapshots=[], last_sequence=6000,
                         name="empty_values")


def many_files():
    # > 1 MiB minimum max_file_size clamp: 6 MiB of input into 1 MiB files
    opts = TableOptions(max_file_size=1 << 20)
    return workloads.l0_l1_job(21, n0=2, n1=2, entries_per_table=12000, options=opts,
                               name="many_files")


def grandparent_cuts():
    job = workloads.l1_l2_at_size(seed=5, scale=0.08, n_l2_tables=8, n_l3_files=200)
    job.name = "grandparent_cuts"
    # small grandparents so that cuts fire often
    for f in job.files:
        if f.level == 3:
            f.file_size = 1 << 20
    return job


def deep_base_levels():
    # files at L+2 and L+3 covering parts of the range: some tombstones stay
    rng = np.random.default_rng(14)
    l0 = [(b"d%06d" % i, 5000 + i, 0 if i % 4 == 0 else 1, rng.bytes(25)) for i in range(3000)]
    l1 = [(b"d%06d" % i, 10 + i, 1, rng.bytes(25)) for i in range(0, 3000, 2)]
    files = [_table(0, 1, l0), _table(1, 2, l1)]
    num = 3
    for lvl, spans in ((2, [(100, 400), (900, 1100)]), (3, [(1500, 2200)]), (5, [(2800, 2900)])):
        for a, b in spans:
            files.append(FileMeta(level=lvl, number=num,
                                  smallest=internal_key(b"d%06d" % a, 1, 1),
                                  largest=internal_key(b"d%06d" % b, 1, 1), file_size=3 << 20))
            num += 1
    return CompactionJob(level=0, files=files, snapshots=[], last_sequence=9000,
                         name="deep_base_levels")


def long_keys():
    rng = np.random.default_rng(15)
    items = [(b"L" * 200 + b"%06d" % i + bytes(rng.integers(0, 256, 300, dtype=np.uint8)),
              1 + i, 1, rng.bytes(int(rng.integers(0, 2000)))) for i in range(800)]
    return CompactionJob(level=0, files=[_table(0, 1, items)], snapshots=[], last_sequence=900,
                         name="long_keys")


def all_cases():
    return [
        single_entry(), all_dropped(),
        options_variant(restart_interval=1), options_variant(restart_interval=2),
        options_variant(block_size=1024), options_variant(block_size=65536),
        options_variant(bits_per_key=0), options_variant(bits_per_key=1),
        options_variant(bits_per_key=20), unparseable_keys(), ff_keys_and_prefixes(),
        snapshot_versions(), identical_internal_keys(), empty_values(), many_files(),
        grandparent_cuts(), deep_base_levels(), long_keys(),
    ]
