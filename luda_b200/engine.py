"""ctypes binding of the engine's C ABI (``include/luda_b200.h``).

``Engine.compact(job)`` is the Python-side counterpart of one
``DBImpl::DoCompactionWork`` call (db/db_impl.cc:1060): it builds the
descriptor from a :class:`luda_b200.job.CompactionJob` exactly as a patched
LevelDB host would from its ``Compaction`` object, calls ``lc_compact`` and
returns the output files with their smallest/largest internal keys.

The shared library is required: if ``libluda_b200.so`` is missing or cannot be
loaded the constructor raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import weakref
from typing import List, Optional, Sequence

import numpy as np

from .job import CompactionJob, Entries, TableOptions

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libluda_b200.so")

_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)

LC_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "corruption", 3: "cuda error", 4: "out of memory",
          5: "over device budget", 6: "timeout", 7: "unsupported", 8: "shutting down"}


class LcConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("device_budget_bytes", C.c_uint64),
                ("max_inflight_jobs", C.c_int32), ("flags", C.c_uint32),
                ("max_batch_jobs", C.c_int32), ("max_batch_bytes", C.c_uint64),
                ("pinned_reserve_bytes", C.c_uint64)]


class LcEngineStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "batches", "jobs", "graph_captures", "graph_replays", "direct_tails", "pinned_bytes",
        "pinned_free_bytes", "inflight_bytes", "queued_jobs", "block_takes", "block_take_us",
        "staging_grows", "pinned_slab_grows", "setup_us_max", "exact_reruns", "scratch_bytes",
        "scratch_free_bytes", "scratch_peak_bytes", "scratch_slab_grows", "device_out_bytes",
        "device_out_free_bytes", "device_out_peak_bytes", "device_out_slab_grows")]


class LcTuning(C.Structure):
    _fields_ = [("ctas_per_job", C.c_uint32), ("merge_items", C.c_uint32),
                ("merge_threads", C.c_uint32)]


class LcTable(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_uint64)]


class LcFileRange(C.Structure):
    _fields_ = [("smallest", _u8p), ("smallest_len", C.c_uint32), ("largest", _u8p),
                ("largest_len", C.c_uint32), ("file_size", C.c_uint64), ("level", C.c_int32)]


class LcTableOptions(C.Structure):
    _fields_ = [("block_size", C.c_uint32), ("restart_interval", C.c_uint32),
                ("bits_per_key", C.c_int32), ("max_file_size", C.c_uint64)]


class LcJobDesc(C.Structure):
    _fields_ = [("level", C.c_int32), ("n_tables", C.c_int32), ("tables", C.POINTER(LcTable)),
                ("n_runs", C.c_int32), ("run_table_count", C.POINTER(C.c_int32)),
                ("n_grandparents", C.c_int32), ("grandparents", C.POINTER(LcFileRange)),
                ("n_base_files", C.c_int32), ("base_files", C.POINTER(LcFileRange)),
                ("smallest_snapshot", C.c_uint64), ("options", LcTableOptions),
                ("inputs_on_device", C.c_int32), ("outputs_on_device", C.c_int32),
                ("verify_checksums", C.c_int32), ("keep_decoded", C.c_int32),
                ("decoded", C.POINTER(C.c_void_p))]


class LcJobOut(C.Structure):
    _fields_ = [("n_files", C.c_int32), ("data", C.c_void_p), ("file_offset", _u64p),
                ("file_size", _u64p), ("file_entries", _u64p), ("key_bytes", _u8p),
                ("smallest_offset", _u64p), ("smallest_len", _u32p), ("largest_offset", _u64p),
                ("largest_len", _u32p), ("bytes_in", C.c_uint64), ("bytes_out", C.c_uint64),
                ("entries_in", C.c_uint64), ("entries_out", C.c_uint64), ("device_ms", C.c_double),
                ("kernel_launches", C.c_uint32), ("n_phases", C.c_uint32),
                ("phase_name", C.POINTER(C.c_char_p)), ("phase_ms", C.POINTER(C.c_float)),
                ("key_bytes_in", C.c_uint64), ("value_bytes_out", C.c_uint64),
                ("key_bytes_out", C.c_uint64), ("device_data", C.c_void_p),
                ("batch_jobs", C.c_uint32), ("queue_ms", C.c_double),
                ("decoded", C.POINTER(C.c_void_p)), ("decoded_inputs", C.c_uint32)]

LC_FLAG_PHASE_TIMING = 1
LC_FLAG_NO_GRAPHS = 2


EXPORTS = ["lc_engine_create", "lc_engine_destroy", "lc_job_submit", "lc_job_wait",
           "lc_job_result", "lc_job_release", "lc_compact", "lc_build_table", "lc_last_error",
           "lc_status_string", "lc_version", "lc_crc32c", "lc_crc32c_noalloc",
           "lc_compact_batch", "lc_get_tuning", "lc_set_tuning", "lc_autotune",
           "lc_job_wait_any", "lc_engine_get_stats", "lc_estimate_device_bytes"]


class LcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads the engine library (raises if it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run luda_b200/build.py")
    l = C.CDLL(path)
    l.lc_engine_create.argtypes = [C.POINTER(LcConfig), C.POINTER(C.c_void_p)]
    l.lc_engine_create.restype = C.c_int
    l.lc_engine_destroy.argtypes = [C.c_void_p]
    l.lc_engine_destroy.restype = None
    l.lc_job_submit.argtypes = [C.c_void_p, C.POINTER(LcJobDesc), C.POINTER(C.c_void_p)]
    l.lc_job_submit.restype = C.c_int
    l.lc_job_wait.argtypes = [C.c_void_p, C.c_int64]
    l.lc_job_wait.restype = C.c_int
    l.lc_job_result.argtypes = [C.c_void_p, C.POINTER(LcJobOut)]
    l.lc_job_result.restype = C.c_int
    l.lc_job_release.argtypes = [C.c_void_p]
    l.lc_job_release.restype = None
    l.lc_compact.argtypes = [C.c_void_p, C.POINTER(LcJobDesc), C.POINTER(LcJobOut),
                             C.POINTER(C.c_void_p)]
    l.lc_compact.restype = C.c_int
    l.lc_estimate_device_bytes.argtypes = [C.POINTER(LcJobDesc), C.POINTER(C.c_uint64)]
    l.lc_estimate_device_bytes.restype = C.c_int
    l.lc_engine_get_stats.argtypes = [C.c_void_p, C.POINTER(LcEngineStats)]
    l.lc_engine_get_stats.restype = C.c_int
    l.lc_job_wait_any.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, C.c_int64,
                                  C.POINTER(C.c_int32)]
    l.lc_job_wait_any.restype = C.c_int
    l.lc_compact_batch.argtypes = [C.c_void_p, C.c_int32, C.POINTER(LcJobDesc),
                                   C.POINTER(C.c_void_p)]
    l.lc_compact_batch.restype = C.c_int
    l.lc_get_tuning.argtypes = [C.c_void_p, C.POINTER(LcTuning)]
    l.lc_get_tuning.restype = C.c_int
    l.lc_set_tuning.argtypes = [C.c_void_p, C.POINTER(LcTuning)]
    l.lc_set_tuning.restype = C.c_int
    l.lc_autotune.argtypes = [C.c_void_p, C.c_int32, C.POINTER(LcJobDesc), C.c_int32,
                              C.POINTER(LcTuning)]
    l.lc_autotune.restype = C.c_int
    l.lc_build_table.argtypes = [C.c_void_p, C.POINTER(LcTableOptions), C.c_int64, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                 C.POINTER(LcJobOut), C.POINTER(C.c_void_p)]
    l.lc_build_table.restype = C.c_int
    l.lc_last_error.argtypes = []
    l.lc_last_error.restype = C.c_char_p
    l.lc_status_string.argtypes = [C.c_int]
    l.lc_status_string.restype = C.c_char_p
    l.lc_crc32c.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(C.c_uint32)]
    l.lc_crc32c.restype = C.c_int
    l.lc_version.argtypes = []
    l.lc_version.restype = C.c_char_p
    _lib = l
    return l


@dataclasses.dataclass
class OutputFile:
    data: object  # bytes-like view of the file (zero copy while the result lives)
    smallest: bytes
    largest: bytes
    entries: int
    decoded: Optional[int] = None  # lc_decoded handle (keep_decoded), valid while the result lives


@dataclasses.dataclass
class CompactionResult:
    files: List[OutputFile]
    bytes_in: int
    bytes_out: int
    entries_in: int
    entries_out: int
    device_ms: float
    device_ptr: Optional[int] = None  # output base in device memory (outputs_on_device 1 or 2)
    file_offsets: Optional[List[int]] = None
    kernel_launches: int = 0
    phase_ms: Optional[dict] = None
    key_bytes_in: int = 0
    value_bytes_out: int = 0
    key_bytes_out: int = 0
    batch_jobs: int = 1
    queue_ms: float = 0.0
    _handle: object = None
    decoded_inputs: int = 0  # input tables read from their decoded form

    def release(self):
        """Frees the job's output buffers (host pinned or device)."""
        if self._handle is not None:
            self._handle.release()
            self._handle = None

    def file_bytes(self) -> List[bytes]:
        return [bytes(f.data) for f in self.files]


class _JobHandle:
    def __init__(self, lib, h, eng=None):
        self.lib, self.h = lib, h
        if eng is not None:
            eng._live.add(self)

    def release(self):
        if self.h is not None:
            self.lib.lc_job_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def _u8(b) -> np.ndarray:
    """A uint8 array over b without copying when b is a contiguous buffer."""
    if isinstance(b, np.ndarray):
        return np.ascontiguousarray(b, dtype=np.uint8)
    if not len(b):
        return np.zeros(1, np.uint8)
    try:
        return np.frombuffer(b, np.uint8)
    except (TypeError, ValueError):
        return np.frombuffer(bytes(b), np.uint8)


class _Keep:
    def __init__(self):
        self.objs = []

    def u8(self, b):
        a = _u8(b)
        self.objs.append(a)
        return a.ctypes.data_as(_u8p)


def table_options(o: TableOptions) -> LcTableOptions:
    return LcTableOptions(o.block_size, o.restart_interval, o.bits_per_key, o.max_file_size)


def make_desc(job: CompactionJob, keep: _Keep, device_tables: Optional[Sequence[int]] = None,
              outputs_on_device: int = 0, verify_checksums: bool = False,
              keep_decoded: bool = False, decoded: Optional[Sequence[Optional[int]]] = None
              ) -> LcJobDesc:
    """The descriptor a patched DoCompactionWork would build from its
    Compaction: runs in MakeInputIterator order, grandparents_, and every file
    at levels >= L+2 for the base-level test.  ``decoded``: per input table (in
    the same order as ``device_tables``) the ``lc_decoded`` handle of its
    decoded form, or None."""
    runs = job.runs()
    tables = [f for r in runs for f in r]
    t_arr = (LcTable * max(1, len(tables)))()
    for i, f in enumerate(tables):
        if device_tables is not None:
            t_arr[i].data = device_tables[i]
        else:
            a = _u8(f.data)
            keep.objs.append(a)
            t_arr[i].data = a.ctypes.data
        t_arr[i].size = len(f.data) if f.data is not None else f.file_size
    rc = (C.c_int32 * max(1, len(runs)))(*[len(r) for r in runs])

    def ranges(fs):
        arr = (LcFileRange * max(1, len(fs)))()
        for i, f in enumerate(fs):
            arr[i].smallest = keep.u8(f.smallest)
            arr[i].smallest_len = len(f.smallest)
            arr[i].largest = keep.u8(f.largest)
            arr[i].largest_len = len(f.largest)
            arr[i].file_size = f.file_size
            arr[i].level = f.level
        return arr

    gp, base = job.grandparents(), job.base_files()
    gpa, ba = ranges(gp), ranges(base)
    keep.objs += [t_arr, rc, gpa, ba]
    dec = None
    if decoded is not None and any(decoded):
        dec = (C.c_void_p * max(1, len(tables)))(*[d or None for d in decoded])
        keep.objs.append(dec)
    return LcJobDesc(job.level, len(tables), t_arr, len(runs), rc, len(gp), gpa, len(base), ba,
                     job.smallest_snapshot(), table_options(job.options),
                     1 if device_tables is not None else 0, int(outputs_on_device),
                     1 if verify_checksums else 0, 1 if keep_decoded else 0,
                     C.cast(dec, C.POINTER(C.c_void_p)) if dec is not None else None)


def _result(out: LcJobOut, outputs_on_device) -> CompactionResult:
    """outputs_on_device: 0/False host bytes, 1/True device only, 2 both."""
    on_device = int(outputs_on_device) == 1
    files = []
    offs = []
    whole = None
    if not on_device and out.bytes_out:
        whole = np.ctypeslib.as_array(C.cast(out.data, _u8p), shape=(out.bytes_out,))
    for i in range(out.n_files):
        off, size = out.file_offset[i], out.file_size[i]
        offs.append(off)
        data = b"" if on_device else memoryview(whole[off:off + size])
        sm = C.string_at(C.addressof(out.key_bytes.contents) + out.smallest_offset[i],
                         out.smallest_len[i])
        lg = C.string_at(C.addressof(out.key_bytes.contents) + out.largest_offset[i],
                         out.largest_len[i])
        dec = out.decoded[i] if out.decoded else None
        files.append(OutputFile(data, sm, lg, int(out.file_entries[i]), dec))
    phases = {out.phase_name[i].decode(): out.phase_ms[i] for i in range(out.n_phases)}
    return CompactionResult(files, out.bytes_in, out.bytes_out, out.entries_in, out.entries_out,
                            out.device_ms, out.device_data, offs,
                            out.kernel_launches, phases or None, out.key_bytes_in,
                            out.value_bytes_out, out.key_bytes_out, out.batch_jobs,
                            out.queue_ms, decoded_inputs=out.decoded_inputs)


class Engine:
    """One CUDA device's compaction engine (``lc_engine``)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_inflight: int = 4,
                 phase_timing: bool = False, graphs: bool = True, max_batch: int = 0,
                 max_batch_bytes: int = 0, pinned_reserve: int = 0):
        self.lib = load_library()
        flags = (LC_FLAG_PHASE_TIMING if phase_timing else 0) | (0 if graphs else LC_FLAG_NO_GRAPHS)
        cfg = LcConfig(device, budget_bytes, max_inflight, flags, max_batch, max_batch_bytes,
                       pinned_reserve)
        h = C.c_void_p()
        st = self.lib.lc_engine_create(C.byref(cfg), C.byref(h))
        if st != LC_OK:
            raise LcError(st, self.lib.lc_last_error().decode())
        self.h = h
        self._live = weakref.WeakSet()

    def close(self):
        if getattr(self, "h", None):
            for jh in list(self._live):
                jh.release()
            self.lib.lc_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != LC_OK:
            raise LcError(st, self.lib.lc_last_error().decode())

    def prepare(self, job: CompactionJob, device_tables: Optional[Sequence[int]] = None,
                outputs_on_device: int = 0, verify_checksums: bool = False,
                keep_decoded: bool = False,
                decoded: Optional[Sequence[Optional[int]]] = None) -> "PreparedJob":
        """Builds the C descriptor once, for repeated runs of the same job.
        ``verify_checksums`` checks every input data block's CRC first
        (LevelDB's paranoid_checks on compaction inputs).  ``keep_decoded``
        keeps the outputs' decoded entries on the device (``OutputFile.decoded``);
        ``decoded`` gives, per device table, such a handle or None."""
        keep = _Keep()
        return PreparedJob(make_desc(job, keep, device_tables, outputs_on_device,
                                     verify_checksums, keep_decoded, decoded), keep,
                           outputs_on_device)

    def run(self, p: "PreparedJob") -> CompactionResult:
        out = LcJobOut()
        jh = C.c_void_p()
        self._check(self.lib.lc_compact(self.h, C.byref(p.desc), C.byref(out), C.byref(jh)))
        res = _result(out, p.outputs_on_device)
        res._handle = _JobHandle(self.lib, jh, self)
        return res

    def run_raw(self, p: "PreparedJob"):
        """``lc_compact`` on a prepared descriptor, returning the raw job
        handle (release with :meth:`release_raw`) and the ``lc_job_out``: the
        bare C-ABI call, without building Python result objects."""
        out = LcJobOut()
        jh = C.c_void_p()
        self._check(self.lib.lc_compact(self.h, C.byref(p.desc), C.byref(out), C.byref(jh)))
        return jh, out

    def release_raw(self, jh) -> None:
        self.lib.lc_job_release(jh)

    def compact(self, job: CompactionJob, device_tables: Optional[Sequence[int]] = None,
                outputs_on_device: int = 0, verify_checksums: bool = False) -> CompactionResult:
        return self.run(self.prepare(job, device_tables, outputs_on_device, verify_checksums))

    @staticmethod
    def _desc_array(prepared: Sequence["PreparedJob"]):
        arr = (LcJobDesc * max(1, len(prepared)))()
        for i, p in enumerate(prepared):
            arr[i] = p.desc
        return arr

    def run_batch(self, prepared: Sequence["PreparedJob"], errors: str = "raise") -> list:
        """Runs the prepared jobs as batches (``lc_compact_batch``); every
        result is byte-identical to running the job alone.  With
        ``errors="raise"`` the first failed job raises (after every handle is
        released); with ``errors="return"`` a failed job's slot holds its
        :class:`LcError` and the other results are returned."""
        n = len(prepared)
        arr = self._desc_array(prepared)
        hs = (C.c_void_p * max(1, n))()
        st = self.lib.lc_compact_batch(self.h, n, arr, hs)
        if st != LC_OK and (errors == "raise" or not any(hs[i] for i in range(n))):
            msg = self.lib.lc_last_error().decode()
            for i in range(n):
                if hs[i]:
                    self.lib.lc_job_release(hs[i])
            raise LcError(st, msg)
        res = []
        for i in range(n):
            out = LcJobOut()
            jst = self.lib.lc_job_result(hs[i], C.byref(out))
            if jst != LC_OK:
                res.append(LcError(jst, self.lib.lc_last_error().decode()))
                self.lib.lc_job_release(hs[i])
                continue
            r = _result(out, prepared[i].outputs_on_device)
            r._handle = _JobHandle(self.lib, C.c_void_p(hs[i]), self)
            res.append(r)
        return res

    def compact_batch(self, jobs: Sequence[CompactionJob],
                      outputs_on_device: int = 0) -> List[CompactionResult]:
        return self.run_batch([self.prepare(j, None, outputs_on_device) for j in jobs])

    def estimate_device_bytes(self, p: "PreparedJob") -> int:
        """Device bytes the job is admitted with (``lc_estimate_device_bytes``)."""
        v = C.c_uint64()
        self._check(self.lib.lc_estimate_device_bytes(C.byref(p.desc), C.byref(v)))
        return v.value

    def stats(self) -> dict:
        """Engine counters (``lc_engine_get_stats``)."""
        st = LcEngineStats()
        self._check(self.lib.lc_engine_get_stats(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in LcEngineStats._fields_}

    def wait_any(self, jobs: Sequence["AsyncJob"], timeout_s: float = -1.0) -> Optional[int]:
        """Index of a finished job among ``jobs`` (``lc_job_wait_any``), or
        None when ``timeout_s`` passes first."""
        arr = (C.c_void_p * max(1, len(jobs)))(*[j.h for j in jobs])
        idx = C.c_int32(-1)
        st = self.lib.lc_job_wait_any(self.h, arr, len(jobs),
                                      int(timeout_s * 1e9) if timeout_s >= 0 else -1,
                                      C.byref(idx))
        if st == 6:
            return None
        self._check(st)
        return idx.value

    def tuning(self) -> dict:
        t = LcTuning()
        self._check(self.lib.lc_get_tuning(self.h, C.byref(t)))
        return {"ctas_per_job": t.ctas_per_job, "merge_items": t.merge_items,
                "merge_threads": t.merge_threads}

    def set_tuning(self, ctas_per_job: int = 0, merge_items: int = 8, merge_threads: int = 256):
        t = LcTuning(ctas_per_job, merge_items, merge_threads)
        self._check(self.lib.lc_set_tuning(self.h, C.byref(t)))

    def autotune(self, prepared: Sequence["PreparedJob"], repeats: int = 2) -> dict:
        """Times candidate launch settings on these jobs (``lc_autotune``) and
        keeps the fastest for the engine."""
        arr = self._desc_array(prepared)
        t = LcTuning()
        self._check(self.lib.lc_autotune(self.h, len(prepared), arr, repeats, C.byref(t)))
        return {"ctas_per_job": t.ctas_per_job, "merge_items": t.merge_items,
                "merge_threads": t.merge_threads}

    def submit_prepared(self, p: "PreparedJob") -> "AsyncJob":
        jh = C.c_void_p()
        self._check(self.lib.lc_job_submit(self.h, C.byref(p.desc), C.byref(jh)))
        return AsyncJob(self, jh, p.keep, p.outputs_on_device)

    def submit(self, job: CompactionJob) -> "AsyncJob":
        keep = _Keep()
        d = make_desc(job, keep)
        jh = C.c_void_p()
        self._check(self.lib.lc_job_submit(self.h, C.byref(d), C.byref(jh)))
        return AsyncJob(self, jh, keep)

    def crc32c(self, data=None, device_ptr: Optional[int] = None, n: int = 0) -> int:
        """Masked CRC32C (LevelDB block-trailer form) of host bytes or of n
        bytes at a device pointer."""
        out = C.c_uint32()
        if device_ptr is not None:
            self._check(self.lib.lc_crc32c(self.h, device_ptr, n, 1, C.byref(out)))
        else:
            a = _u8(data)
            self._check(self.lib.lc_crc32c(self.h, a.ctypes.data, len(data), 0, C.byref(out)))
        return out.value

    def build_table(self, entries: Entries, options: TableOptions) -> bytes:
        keys = _u8(entries.keys)
        vals = _u8(entries.vals)
        ko = np.ascontiguousarray(entries.koffs, np.uint64)
        vo = np.ascontiguousarray(entries.voffs, np.uint64)
        opt = table_options(options)
        out = LcJobOut()
        jh = C.c_void_p()
        self._check(self.lib.lc_build_table(self.h, C.byref(opt), entries.n, keys.ctypes.data,
                                            ko.ctypes.data, vals.ctypes.data, vo.ctypes.data, 0,
                                            C.byref(out), C.byref(jh)))
        try:
            assert out.n_files == 1
            return C.string_at(out.data + out.file_offset[0], out.file_size[0])
        finally:
            self.lib.lc_job_release(jh)


@dataclasses.dataclass
class PreparedJob:
    desc: LcJobDesc
    keep: object
    outputs_on_device: int


class AsyncJob:
    def __init__(self, eng: Engine, h, keep, outputs_on_device: int = 0):
        self.eng, self.h, self.keep = eng, h, keep
        self.outputs_on_device = outputs_on_device

    def wait(self, timeout_s: float = -1.0) -> CompactionResult:
        lib = self.eng.lib
        st = lib.lc_job_wait(self.h, int(timeout_s * 1e9) if timeout_s >= 0 else -1)
        if st == 6:
            raise TimeoutError("job not finished")
        try:
            self.eng._check(st)
            out = LcJobOut()
            self.eng._check(lib.lc_job_result(self.h, C.byref(out)))
        except Exception:
            lib.lc_job_release(self.h)
            self.h = None
            raise
        res = _result(out, self.outputs_on_device)
        res._handle = _JobHandle(lib, self.h, self.eng)
        self.h = None
        return res
