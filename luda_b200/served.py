"""Served compaction: a request loop over simulated LevelDB instances.

A random-fill write stream (16-byte keys uniform over 2^26, 100-byte values)
is cut into 4 MiB memtables; each flush adds a level-0 table to one of several
simulated databases.  Every database picks its compactions the way
``VersionSet::PickCompaction`` does (db/version_set.cc:1270-1318, scores from
``VersionSet::Finalize`` :1012-1047): level 0 by file count against
``kL0_CompactionTrigger`` (db/dbformat.h:25), other levels by bytes against
``MaxBytesForLevel`` (db/version_set.cc:43-53), the first file after the
level's compaction pointer, level-0 inputs widened to every overlapping
level-0 file (``GetOverlappingInputs`` :519-559), the overlapping files of
the next level (``SetupOtherInputs`` :1360-1420, without the widening step)
and the grandparents two levels down.  Like LevelDB, a database runs one
compaction at a time and stops taking flushes at ``kL0_StopWritesTrigger``
level-0 files (db/dbformat.h:31).

The loop keeps many databases' compactions in flight on one engine:

* ``mode="served"`` -- jobs go through the engine's asynchronous entry
  points (continuous batching, admission against the device budget).  A new
  level-0 table is copied to the device once when it arrives; every output is
  kept on the device (``outputs_on_device=2``) beside its host copy, so a job
  whose inputs were written by earlier jobs reads them from HBM and crosses
  PCIe only to persist its own outputs.
* ``mode="plain"`` -- the drop-in as LevelDB would call it: one compaction at
  a time (an engine with one worker and batches of one), inputs copied from
  host memory, outputs copied back.

Both record each job's latency (from the moment it was submitted to the
engine to its completion), its input bytes (the reference's
``CompactionStats::bytes_read``, db/db_impl.cc:1203-1207) and the makespan.
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from typing import Callable, List, Optional, Sequence

import numpy as np

from .job import CompactionJob, Entries, FileMeta, TableOptions, icmp_key

KEY_SPACE = 1 << 26
VALUE_BYTES = 100
MEMTABLE_BYTES = 4 << 20
L0_COMPACTION_TRIGGER = 4  # db/dbformat.h:25
L0_STOP_WRITES_TRIGGER = 12  # db/dbformat.h:31
NUM_LEVELS = 7


def max_bytes_for_level(level: int) -> float:
    """db/version_set.cc:43-53 (level >= 1)."""
    r = 10.0 * 1048576.0
    while level > 1:
        r *= 10
        level -= 1
    return r


def memtable_entries(rng: np.random.Generator, seq0: int,
                     n: Optional[int] = None) -> Entries:
    """One memtable of the random-fill stream, in internal-key order: n puts
    (about 4 MiB of 16-byte keys + 8-byte tags + 100-byte values) with
    sequence numbers seq0+1 .. seq0+n in arrival order."""
    if n is None:
        n = MEMTABLE_BYTES // (16 + 8 + VALUE_BYTES)
    ids = rng.integers(0, KEY_SPACE, size=n, dtype=np.int64)
    seqs = np.arange(seq0 + 1, seq0 + n + 1, dtype=np.uint64)
    # user key ascending, then sequence descending (db/dbformat.cc:51-67)
    order = np.lexsort((-seqs.astype(np.int64), ids))
    ids, seqs = ids[order], seqs[order]
    digits = np.zeros((n, 16), np.uint8)
    v = ids.copy()
    for c in range(15, -1, -1):
        digits[:, c] = 48 + (v % 10)
        v //= 10
    tags = (seqs << np.uint64(8)) | np.uint64(1)  # kTypeValue
    keys = np.concatenate([digits, tags.view(np.uint8).reshape(n, 8)], axis=1).reshape(-1)
    koffs = np.arange(n + 1, dtype=np.uint64) * np.uint64(24)
    vals = rng.integers(0, 256, size=n * VALUE_BYTES, dtype=np.uint8)
    voffs = np.arange(n + 1, dtype=np.uint64) * np.uint64(VALUE_BYTES)
    return Entries(keys, koffs, vals, voffs)


@dataclasses.dataclass
class Flush:
    """A level-0 table ready to be added to database ``db`` at time ``t``."""
    t: float
    db: int
    data: object  # table bytes (host)
    smallest: bytes
    largest: bytes
    last_seq: int


@dataclasses.dataclass(eq=False)
class SimTable:
    number: int
    level: int
    smallest: bytes
    largest: bytes
    size: int
    host: object = None  # table bytes in host memory (the persisted copy)
    dev: int = 0  # device address of the same bytes, 0 if not resident
    owner: object = None  # _Owner keeping host/device memory alive
    ready: Optional[Callable[[], None]] = None  # waits until the device copy exists
    dec: Optional[int] = None  # handle of its decoded entries on the device (outputs of jobs)


class _Owner:
    """Keeps one job result (or one upload) alive while any of its tables is
    still in a database."""

    def __init__(self, obj, count: int, release: Callable[[object], None]):
        self.obj, self.count, self._release = obj, count, release

    def drop(self):
        self.count -= 1
        if self.count == 0 and self.obj is not None:
            self._release(self.obj)
            self.obj = None


def _ukey(ikey: bytes) -> bytes:
    return ikey[:-8]


class SimDB:
    """The version state of one database (files per level, compaction
    pointers, sequence numbers) and LevelDB's choice of the next compaction."""

    def __init__(self, index: int, options: TableOptions, level_scale: float = 1.0):
        self.index = index
        self.options = options
        self.level_scale = level_scale  # < 1 shrinks the level size targets (small tests)
        self.levels: List[List[SimTable]] = [[] for _ in range(NUM_LEVELS)]
        self.compact_pointer: List[Optional[bytes]] = [None] * NUM_LEVELS
        self.next_number = 1
        self.last_seq = 0
        self.busy = False
        self.pending: deque = deque()  # flushes held back by the stop trigger

    def new_number(self) -> int:
        n = self.next_number
        self.next_number += 1
        return n

    def add_l0(self, t: SimTable, last_seq: int):
        self.levels[0].append(t)
        self.last_seq = max(self.last_seq, last_seq)

    def level_bytes(self, level: int) -> int:
        return sum(t.size for t in self.levels[level])

    def score(self):
        """VersionSet::Finalize: the level with the highest score."""
        best, best_level = -1.0, -1
        for level in range(NUM_LEVELS - 1):
            if level == 0:
                s = len(self.levels[0]) / float(L0_COMPACTION_TRIGGER)
            else:
                s = self.level_bytes(level) / (max_bytes_for_level(level) * self.level_scale)
            if s > best:
                best, best_level = s, level
        return best, best_level

    def overlapping(self, level: int, begin: Optional[bytes], end: Optional[bytes]):
        """Version::GetOverlappingInputs over user keys; on level 0 the range
        grows with every overlapping file and the search restarts."""
        files = self.levels[level]
        ub = _ukey(begin) if begin is not None else None
        ue = _ukey(end) if end is not None else None
        out = []
        i = 0
        while i < len(files):
            f = files[i]
            i += 1
            fs, fl = _ukey(f.smallest), _ukey(f.largest)
            if ub is not None and fl < ub:
                continue
            if ue is not None and fs > ue:
                continue
            out.append(f)
            if level == 0:
                if ub is not None and fs < ub:
                    ub, out, i = fs, [], 0
                elif ue is not None and fl > ue:
                    ue, out, i = fl, [], 0
        return out

    @staticmethod
    def _range(files):
        sm = min((f.smallest for f in files), key=icmp_key)
        lg = max((f.largest for f in files), key=icmp_key)
        return sm, lg

    def pick(self):
        """(level, inputs0, inputs1, grandparents) or None."""
        score, level = self.score()
        if score < 1.0:
            return None
        files = sorted(self.levels[level], key=lambda f: (icmp_key(f.smallest), f.number)) \
            if level > 0 else list(self.levels[0])
        ptr = self.compact_pointer[level]
        first = None
        for f in files:
            if ptr is None or icmp_key(f.largest) > icmp_key(ptr):
                first = f
                break
        if first is None:
            first = files[0]
        inputs0 = [first]
        if level == 0:
            sm, lg = self._range(inputs0)
            inputs0 = self.overlapping(0, sm, lg)
        sm, lg = self._range(inputs0)
        inputs1 = self.overlapping(level + 1, sm, lg)
        all_sm, all_lg = self._range(inputs0 + inputs1)
        gp = self.overlapping(level + 2, all_sm, all_lg) if level + 2 < NUM_LEVELS else []
        self.compact_pointer[level] = lg
        return level, inputs0, inputs1, gp

    def job(self, level, inputs0, inputs1) -> CompactionJob:
        """The compaction as the engine's job model sees it: inputs, the
        grandparents' level and every deeper level (for IsBaseLevelForKey)."""
        files = []
        for t in inputs0 + inputs1:
            fm = FileMeta(t.level, t.number, t.smallest, t.largest, t.size, None, None)
            fm.sim = t
            files.append(fm)
        for lvl in range(level + 2, NUM_LEVELS):
            for t in self.levels[lvl]:
                fm = FileMeta(t.level, t.number, t.smallest, t.largest, t.size, None, None)
                fm.sim = t
                files.append(fm)
        return CompactionJob(level, files, [], self.last_seq, self.options,
                             name=f"db{self.index}_L{level}")

    def install(self, level, inputs0, inputs1, outputs: Sequence[SimTable]):
        """VersionEdit: delete the inputs, add the outputs at level+1."""
        gone0 = set(id(t) for t in inputs0)
        gone1 = set(id(t) for t in inputs1)
        self.levels[level] = [t for t in self.levels[level] if id(t) not in gone0]
        self.levels[level + 1] = [t for t in self.levels[level + 1] if id(t) not in gone1]
        self.levels[level + 1].extend(outputs)
        self.levels[level + 1].sort(key=lambda t: icmp_key(t.smallest))
        for t in list(inputs0) + list(inputs1):
            if t.owner is not None:
                t.owner.drop()

    def check_levels(self):
        """Levels >= 1 hold disjoint, ordered key ranges."""
        for lvl in range(1, NUM_LEVELS):
            fs = self.levels[lvl]
            for a, b in zip(fs, fs[1:]):
                assert _ukey(a.largest) < _ukey(b.smallest), (self.index, lvl)


def make_flushes(n_db: int, flushes_per_db: int, build_table: Callable, seed: int = 3,
                 options: Optional[TableOptions] = None, entries_per_flush: Optional[int] = None,
                 ) -> List[List[Flush]]:
    """Per database, its level-0 tables in write order (times filled in by
    ``schedule``); tables are encoded with ``build_table(entries, options)``."""
    options = options or TableOptions()
    out = []
    for d in range(n_db):
        rng = np.random.default_rng(seed * 1000 + d)
        seq = 0
        fl = []
        for _ in range(flushes_per_db):
            e = memtable_entries(rng, seq, entries_per_flush)
            seq += e.n
            data = bytes(build_table(e, options))
            fl.append(Flush(0.0, d, data, e.key(0), e.key(e.n - 1), seq))
        out.append(fl)
    return out


def schedule(flushes: List[List[Flush]], rate_per_s: Optional[float], seed: int = 11
             ) -> List[Flush]:
    """Merges the databases' flush streams into one arrival sequence:
    Poisson arrivals at ``rate_per_s`` (flushes per second over all
    databases; None: everything at time 0), each arrival going to a database
    drawn uniformly among those with flushes left."""
    rng = np.random.default_rng(seed)
    queues = [deque(f) for f in flushes]
    out, t = [], 0.0
    live = [i for i, q in enumerate(queues) if q]
    while live:
        if rate_per_s:
            t += float(rng.exponential(1.0 / rate_per_s))
        d = live[int(rng.integers(0, len(live)))]
        f = queues[d].popleft()
        out.append(dataclasses.replace(f, t=t))
        live = [i for i, q in enumerate(queues) if q]
    return out


@dataclasses.dataclass
class JobRecord:
    db: int
    level: int
    input_bytes: int
    output_bytes: int
    submit_s: float
    done_s: float
    n_inputs: int
    resident_inputs: int
    decoded_inputs: int = 0  # inputs read from their decoded form (no parse, no decode)
    device_ms: float = 0.0  # the engine's device time for the batch that ran the job
    batch_jobs: int = 1  # jobs in that batch
    queue_ms: float = 0.0  # time in the engine's queue before its batch started
    phase_ms: Optional[dict] = None  # the batch's device time per phase, when the engine times phases
    file_bytes: Optional[List[bytes]] = None  # kept when record_bytes
    job: Optional[CompactionJob] = None  # the job with host copies of its inputs

    @property
    def latency_ms(self) -> float:
        return (self.done_s - self.submit_s) * 1e3


@dataclasses.dataclass
class ServeStats:
    mode: str
    makespan_s: float
    jobs: List[JobRecord]
    h2d_bytes: int
    d2h_bytes: int
    stall_s: float
    flushes: int
    host_submit_s: float = 0.0  # loop time spent picking, describing and submitting jobs
    host_complete_s: float = 0.0  # loop time spent collecting results and installing them
    host_result_s: float = 0.0  # ... of which reading the result
    host_install_s: float = 0.0  # ... of which installing (and releasing consumed tables)
    host_upload_s: float = 0.0  # loop time spent copying new level-0 tables to the device
    longest_turn_ms: float = 0.0  # the longest pass of the loop between two waits

    @property
    def input_bytes(self) -> int:
        return sum(j.input_bytes for j in self.jobs)

    def summary(self) -> dict:
        lat = np.array([j.latency_ms for j in self.jobs]) if self.jobs else np.zeros(1)
        q = np.array([j.queue_ms for j in self.jobs]) if self.jobs else np.zeros(1)
        mib = self.input_bytes / float(1 << 20)
        return {
            "mode": self.mode, "jobs": len(self.jobs), "flushes": self.flushes,
            "input_mib": mib, "makespan_s": self.makespan_s,
            "value": mib / self.makespan_s if self.makespan_s > 0 else None, "unit": "MiB/s",
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()),
            "jobs_by_level": {str(l): sum(1 for j in self.jobs if j.level == l)
                              for l in sorted(set(j.level for j in self.jobs))},
            "decoded_resident_fraction": (sum(j.decoded_inputs for j in self.jobs) /
                                          max(1, sum(j.n_inputs for j in self.jobs))),
            "resident_input_fraction": (sum(j.resident_inputs for j in self.jobs) /
                                        max(1, sum(j.n_inputs for j in self.jobs))),
            "h2d_mib": self.h2d_bytes / float(1 << 20),
            "d2h_mib": self.d2h_bytes / float(1 << 20),
            "write_stall_s": self.stall_s,
            "host_submit_s": self.host_submit_s, "host_complete_s": self.host_complete_s,
            "host_result_s": self.host_result_s, "host_install_s": self.host_install_s,
            "host_upload_s": self.host_upload_s, "longest_turn_ms": self.longest_turn_ms,
            "queue_ms_mean": float(q.mean()), "queue_ms_p99": float(np.percentile(q, 99)),
            "device_ms_mean": float(np.mean([j.device_ms for j in self.jobs])) if self.jobs else 0,
            "batch_jobs_mean": float(np.mean([j.batch_jobs for j in self.jobs])) if self.jobs else 0,
            "slowest": [{"latency_ms": j.latency_ms, "queue_ms": j.queue_ms,
                         "device_ms": j.device_ms, "batch_jobs": j.batch_jobs, "level": j.level,
                         "input_mib": j.input_bytes / float(1 << 20), "submit_s": j.submit_s,
                         "phase_ms": ({k: round(v, 3) for k, v in j.phase_ms.items()}
                                      if j.phase_ms else None)}
                        for j in sorted(self.jobs, key=lambda j: -j.latency_ms)[:4]],
        }


class Server:
    """The request loop.  ``engine`` is a :class:`luda_b200.engine.Engine`
    (or an object with the same ``prepare`` / ``submit_prepared`` /
    ``wait_any`` methods); ``upload(bytes) -> (device address, handle)`` and
    ``free(handle)`` move new level-0 tables to the device in served mode, and
    ``ready(handle)``, when given, waits until an upload that ``upload``
    started asynchronously has finished (called before the first job that
    reads the table is submitted)."""

    def __init__(self, engine, n_db: int, mode: str = "served",
                 options: Optional[TableOptions] = None, upload=None, free=None,
                 record_bytes: bool = False, level_scale: float = 1.0, ready=None,
                 keep_decoded: bool = True):
        assert mode in ("served", "plain")
        # served mode: outputs kept on the device also keep their decoded
        # entries, so that the next level's job skips parsing and decoding them
        self.keep_decoded = keep_decoded and mode == "served"
        self.engine = engine
        self.mode = mode
        self.options = options or TableOptions()
        self.dbs = [SimDB(i, self.options, level_scale) for i in range(n_db)]
        self.upload, self.free, self.ready = upload, free, ready
        self.record_bytes = record_bytes
        self.h2d = 0
        self.d2h = 0

    # -- tables ------------------------------------------------------------
    def _l0_table(self, db: SimDB, f: Flush) -> SimTable:
        t = SimTable(db.new_number(), 0, f.smallest, f.largest, len(f.data), host=f.data)
        if self.mode == "served" and self.upload is not None:
            addr, handle = self.upload(f.data)
            t.dev = addr
            t.owner = _Owner(handle, 1, self.free)
            if self.ready is not None:
                t.ready = lambda h=handle: self.ready(h)
            self.h2d += len(f.data)
        return t

    def _outputs(self, db: SimDB, level: int, res) -> List[SimTable]:
        n = len(res.files)
        owner = _Owner(res, n, lambda r: r.release()) if n else None
        if n == 0:
            res.release()
        out = []
        for i, f in enumerate(res.files):
            dev = 0
            if self.mode == "served" and res.device_ptr:
                dev = int(res.device_ptr) + int(res.file_offsets[i])
            out.append(SimTable(db.new_number(), level + 1, f.smallest, f.largest, len(f.data),
                                host=f.data, dev=dev, owner=owner,
                                dec=getattr(f, "decoded", None) if dev else None))
        self.d2h += res.bytes_out
        return out

    # -- jobs --------------------------------------------------------------
    def _submit(self, db: SimDB, now: Callable[[], float]):
        c = db.pick()
        if c is None:
            return None
        level, in0, in1, _ = c
        job = db.job(level, in0, in1)
        tables = job.input_tables()
        resident = sum(1 for f in tables if f.sim.dev)
        if self.mode == "served" and resident == len(tables):
            for f in tables:
                if f.sim.ready is not None:
                    f.sim.ready()
                    f.sim.ready = None
            decoded = [f.sim.dec for f in tables]
            p = self.engine.prepare(job, device_tables=[f.sim.dev for f in tables],
                                    outputs_on_device=2, keep_decoded=self.keep_decoded,
                                    decoded=decoded if self.keep_decoded else None)
            n_decoded = sum(1 for d in decoded if d) if self.keep_decoded else 0
        else:
            for f in tables:
                f.data = f.sim.host
            served_mode = self.mode == "served"
            p = self.engine.prepare(job, outputs_on_device=2 if served_mode else 0,
                                    keep_decoded=served_mode and self.keep_decoded)
            resident = 0
            n_decoded = 0
            self.h2d += sum(f.file_size for f in tables)
        for f in tables:
            # host copy of the inputs for the record (the live buffers are reused)
            f.data = bytes(f.sim.host) if self.record_bytes else None
        h = self.engine.submit_prepared(p)
        db.busy = True
        rec = JobRecord(db.index, level, sum(f.file_size for f in tables), 0, now(), 0.0,
                        len(tables), resident, job=job if self.record_bytes else None,
                        decoded_inputs=n_decoded)
        return h, (db, level, in0, in1, rec, p)

    def run(self, arrivals: Sequence[Flush], clock=time.perf_counter,
            idle_wait: Callable[[float], None] = time.sleep) -> ServeStats:
        t0 = clock()
        inflight: List = []  # (AsyncJob, context)
        records: List[JobRecord] = []
        stall = 0.0
        t_sub = t_done = t_res = t_inst = t_up = 0.0
        longest = 0.0
        since = lambda: clock() - t0  # noqa: E731
        stalled_since = {}
        i = 0
        n = len(arrivals)
        while i < n or inflight or any(d.pending for d in self.dbs):
            now = clock() - t0
            turn0 = now
            while i < n and arrivals[i].t <= now:
                self.dbs[arrivals[i].db].pending.append(arrivals[i])
                i += 1
            for db in self.dbs:
                while db.pending and len(db.levels[0]) < L0_STOP_WRITES_TRIGGER:
                    f = db.pending.popleft()
                    if db.index in stalled_since:
                        stall += now - stalled_since.pop(db.index)
                    u0 = clock()
                    db.add_l0(self._l0_table(db, f), f.last_seq)
                    t_up += clock() - u0
                if db.pending and db.index not in stalled_since:
                    stalled_since[db.index] = now
                if not db.busy:
                    c0 = clock()
                    s = self._submit(db, since)
                    t_sub += clock() - c0
                    if s is not None:
                        inflight.append(s)
            if not inflight:
                if i < n:
                    idle_wait(max(0.0, arrivals[i].t - (clock() - t0)))
                continue
            timeout = max(0.0, arrivals[i].t - (clock() - t0)) if i < n else -1.0
            longest = max(longest, clock() - t0 - turn0)
            k = self.engine.wait_any([h for h, _ in inflight], timeout)
            if k is None:
                continue
            h, (db, level, in0, in1, rec, p) = inflight.pop(k)
            c0 = clock()
            res = h.wait()
            rec.done_s = c0 - t0
            rec.output_bytes = res.bytes_out
            rec.device_ms = getattr(res, "device_ms", 0.0)
            rec.batch_jobs = getattr(res, "batch_jobs", 1)
            rec.queue_ms = getattr(res, "queue_ms", 0.0)
            rec.phase_ms = getattr(res, "phase_ms", None)
            if self.record_bytes:
                rec.file_bytes = res.file_bytes()
            outs = self._outputs(db, level, res)
            c1 = clock()
            t_res += c1 - c0
            db.install(level, in0, in1, outs)
            t_inst += clock() - c1
            db.busy = False
            records.append(rec)
            t_done += clock() - c0
        return ServeStats(self.mode, clock() - t0, records, self.h2d, self.d2h, stall, n,
                          t_sub, t_done, t_res, t_inst, t_up, longest * 1e3)

    def close(self):
        """Releases every table still held by the databases."""
        for db in self.dbs:
            for lvl in db.levels:
                for t in lvl:
                    if t.owner is not None:
                        t.owner.drop()
                lvl.clear()
