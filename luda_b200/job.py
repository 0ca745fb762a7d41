"""Host-side model of one compaction job.

Mirrors the pieces of the reference's version set that decide what one
``DBImpl::DoCompactionWork`` call sees (db/db_impl.cc:1060): the input files of
level L and L+1 (``Compaction::inputs_``, db/version_set.h:380), the
grandparent files (``Compaction::grandparents_``, filled by
``VersionSet::SetupOtherInputs``, db/version_set.cc:1446-1450), every file at
levels >= L+2 for ``Compaction::IsBaseLevelForKey`` (db/version_set.cc:1535),
and the smallest live snapshot (db/db_impl.cc:1073-1077).

The same job is handed to the GPU engine (through the C ABI in
``include/luda_b200.h``), to the CPU restatement and to the reference build.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional

import numpy as np

K_NUM_LEVELS = 7  # config::kNumLevels (db/dbformat.h:25)
K_MAX_SEQUENCE = (1 << 56) - 1  # db/dbformat.h:65


@dataclasses.dataclass
class TableOptions:
    """The ``Options`` fields that shape table bytes (include/leveldb/options.h)."""

    block_size: int = 4096  # options.h:100
    restart_interval: int = 16  # options.h:105
    bits_per_key: int = 10  # NewBloomFilterPolicy(bits_per_key); <= 0: no filter
    max_file_size: int = 2 << 20  # options.h:115; Compaction::MaxOutputFileSize


@dataclasses.dataclass
class Entries:
    """Sorted internal keys and their values, packed.

    ``keys[koffs[i]:koffs[i+1]]`` is entry i's internal key (user key followed
    by fixed64 ``seq << 8 | type``, db/dbformat.h:94-100); values likewise.
    """

    keys: np.ndarray  # uint8
    koffs: np.ndarray  # uint64, n+1
    vals: np.ndarray  # uint8
    voffs: np.ndarray  # uint64, n+1

    @property
    def n(self) -> int:
        return int(len(self.koffs) - 1)

    def key(self, i: int) -> bytes:
        return self.keys[int(self.koffs[i]):int(self.koffs[i + 1])].tobytes()

    def value(self, i: int) -> bytes:
        return self.vals[int(self.voffs[i]):int(self.voffs[i + 1])].tobytes()

    def nbytes(self) -> int:
        return int(self.koffs[-1] + self.voffs[-1])

    @staticmethod
    def from_lists(keys: List[bytes], vals: List[bytes]) -> "Entries":
        koffs = np.zeros(len(keys) + 1, np.uint64)
        voffs = np.zeros(len(vals) + 1, np.uint64)
        koffs[1:] = np.cumsum([len(k) for k in keys], dtype=np.uint64)
        voffs[1:] = np.cumsum([len(v) for v in vals], dtype=np.uint64)
        kb = np.frombuffer(b"".join(keys), np.uint8) if keys else np.zeros(0, np.uint8)
        vb = np.frombuffer(b"".join(vals), np.uint8) if vals else np.zeros(0, np.uint8)
        return Entries(kb.copy(), koffs, vb.copy(), voffs)

    def slice(self, a: int, b: int) -> "Entries":
        k0, k1 = int(self.koffs[a]), int(self.koffs[b])
        v0, v1 = int(self.voffs[a]), int(self.voffs[b])
        return Entries(self.keys[k0:k1].copy(), (self.koffs[a:b + 1] - k0).astype(np.uint64),
                       self.vals[v0:v1].copy(), (self.voffs[a:b + 1] - v0).astype(np.uint64))


def pack_tag(seq: int, vtype: int) -> bytes:
    """fixed64 little-endian ``seq << 8 | type`` (db/dbformat.cc:15-19)."""
    return struct.pack("<Q", (seq << 8) | vtype)


def internal_key(user_key: bytes, seq: int, vtype: int) -> bytes:
    return user_key + pack_tag(seq, vtype)


def icmp_key(ikey: bytes):
    """Sort key equal to InternalKeyComparator order (db/dbformat.cc:51-67)."""
    tag = struct.unpack("<Q", ikey[-8:])[0]
    return (ikey[:-8], -tag)


@dataclasses.dataclass
class FileMeta:
    """``FileMetaData`` (db/version_edit.h:18-27) plus optional contents."""

    level: int
    number: int
    smallest: bytes
    largest: bytes
    file_size: int = 0
    entries: Optional[Entries] = None  # logical content of an input table
    data: Optional[bytes] = None  # table bytes of an input table


@dataclasses.dataclass
class CompactionJob:
    level: int
    files: List[FileMeta]
    snapshots: List[int]
    last_sequence: int
    options: TableOptions = dataclasses.field(default_factory=TableOptions)
    name: str = "job"

    # -- the version's view ------------------------------------------------
    def level_files(self, level: int) -> List[FileMeta]:
        """Files of one level in the version's order: ``BySmallestKey``
        (db/version_set.cc:593-605), ties broken by file number."""
        fs = [f for f in self.files if f.level == level]
        return sorted(fs, key=lambda f: (icmp_key(f.smallest), f.number))

    def inputs(self, which: int) -> List[FileMeta]:
        return self.level_files(self.level + which)

    def runs(self) -> List[List[FileMeta]]:
        """Merge children in ``VersionSet::MakeInputIterator`` order
        (db/version_set.cc:1237-1268): one child per level-0 file, one
        concatenating child per level >= 1."""
        out = []
        for which in (0, 1):
            fs = self.inputs(which)
            if not fs:
                continue
            if self.level + which == 0:
                out.extend([[f] for f in fs])
            else:
                out.append(fs)
        return out

    def input_tables(self) -> List[FileMeta]:
        return [f for run in self.runs() for f in run]

    def grandparents(self) -> List[FileMeta]:
        """``Version::GetOverlappingInputs(level+2, all_start, all_limit)``
        (db/version_set.cc:519-559; level >= 1 branch), over the whole input
        range (``GetRange2``)."""
        if self.level + 2 >= K_NUM_LEVELS:
            return []
        ins = self.inputs(0) + self.inputs(1)
        if not ins:
            return []
        begin = min((f.smallest for f in ins), key=icmp_key)[:-8]
        end = max((f.largest for f in ins), key=icmp_key)[:-8]
        out = []
        for f in self.level_files(self.level + 2):
            if f.largest[:-8] < begin or f.smallest[:-8] > end:
                continue
            out.append(f)
        return out

    def base_files(self) -> List[FileMeta]:
        """Every file at levels >= L+2, each level in key order: what
        ``Compaction::IsBaseLevelForKey`` walks."""
        out = []
        for lvl in range(self.level + 2, K_NUM_LEVELS):
            out.extend(self.level_files(lvl))
        return out

    def smallest_snapshot(self) -> int:
        """db/db_impl.cc:1073-1077: the oldest snapshot, else LastSequence."""
        if self.snapshots:
            return self.snapshots[0]
        return self.last_sequence

    def input_bytes(self) -> int:
        """Sum of input ``file_size``: what the reference counts as
        ``CompactionStats::bytes_read`` (db/db_impl.cc:1203-1207)."""
        return sum(f.file_size for f in self.input_tables())

    # -- building the input tables -----------------------------------------
    def materialize(self, build_table) -> "CompactionJob":
        """Encodes every input file's entries with ``build_table(entries,
        options) -> bytes`` and fills in ``data`` / ``file_size``."""
        for f in self.files:
            if f.entries is not None and f.data is None:
                f.data = bytes(build_table(f.entries, self.options))
                f.file_size = len(f.data)
        return self
