"""Test infrastructure, not product code.

ctypes front end to the two CPU checkers built by ``oracle/Makefile``:

* ``oracle/_build/liblsm_oracle.so`` -- the C restatement (``lsm_oracle.c``);
* ``oracle/_ref/libluda_ref.so``      -- the reference's own CPU compaction,
  compiled from the reference sources (present only where they were
  available at build time; the built library travels with the repository).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker.  The GPU engine never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liblsm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libluda_ref.so")
# Location of the reference source tree, for building the reference library
# only (the built library travels with the repository; nothing reads the
# sources at run time).  No default: the caller names it.
REF_ROOT = os.environ.get("LUDA_REF_ROOT")

_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)


class LoTable(C.Structure):
    _fields_ = [("data", _u8p), ("size", C.c_uint64)]


class LoFileRange(C.Structure):
    _fields_ = [("smallest", _u8p), ("smallest_len", C.c_uint32),
                ("largest", _u8p), ("largest_len", C.c_uint32),
                ("file_size", C.c_uint64), ("level", C.c_int32)]


class LoJob(C.Structure):
    _fields_ = [("level", C.c_int32), ("n_tables", C.c_int32), ("tables", C.POINTER(LoTable)),
                ("n_runs", C.c_int32), ("run_table_count", C.POINTER(C.c_int32)),
                ("n_grandparents", C.c_int32), ("grandparents", C.POINTER(LoFileRange)),
                ("n_base_files", C.c_int32), ("base_files", C.POINTER(LoFileRange)),
                ("smallest_snapshot", C.c_uint64), ("block_size", C.c_uint32),
                ("restart_interval", C.c_uint32), ("bits_per_key", C.c_int32),
                ("max_file_size", C.c_uint64)]


class RefFile(C.Structure):
    _fields_ = [("data", _u8p), ("size", C.c_uint64), ("level", C.c_int32),
                ("smallest", _u8p), ("smallest_len", C.c_uint32),
                ("largest", _u8p), ("largest_len", C.c_uint32)]


class RefJob(C.Structure):
    _fields_ = [("level", C.c_int32), ("n_files", C.c_int32), ("files", C.POINTER(RefFile)),
                ("n_snapshots", C.c_int32), ("snapshots", _u64p),
                ("last_sequence", C.c_uint64), ("block_size", C.c_uint32),
                ("restart_interval", C.c_uint32), ("bits_per_key", C.c_int32),
                ("max_file_size", C.c_uint64)]


def build(ref: bool = True, ref_root: Optional[str] = None) -> None:
    """Builds the restatement and, when ``ref_root`` (or ``LUDA_REF_ROOT``)
    names an existing reference source tree, the reference library."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    root = ref_root or REF_ROOT
    if ref and root and os.path.isdir(root):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF_ROOT={root}"],
                       check=True)
        # the compiled drop-in and its CPU twin (needs the engine library built)
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "dropin", f"REF_ROOT={root}"],
                       check=True)


_libs = {}


def _bind(lib, prefix):
    def f(name, res, *args):
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = list(args)
    f("crc32c_mask" if prefix == "ref_" else "crc32c_mask", C.c_uint32, C.c_uint32)
    f("hash", C.c_uint32, _u8p, C.c_uint64, C.c_uint32)
    f("build_table", C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_int64, _u8p, _u64p,
      _u8p, _u64p)
    f("buf_data", _u8p, C.c_void_p, _u64p)
    f("buf_free", None, C.c_void_p)
    f("bloom", C.c_void_p, C.c_int, C.c_int, _u8p, _u64p)
    f("separator", C.c_void_p, _u8p, C.c_uint32, _u8p, C.c_uint32)
    f("successor", C.c_void_p, _u8p, C.c_uint32)
    f("result_nfiles", C.c_int, C.c_void_p)
    f("result_file", _u8p, C.c_void_p, C.c_int, _u64p)
    f("result_smallest", _u8p, C.c_void_p, C.c_int, C.POINTER(C.c_uint32))
    f("result_largest", _u8p, C.c_void_p, C.c_int, C.POINTER(C.c_uint32))
    f("result_free", None, C.c_void_p)
    if prefix == "lo_":
        f("crc32c_extend", C.c_uint32, C.c_uint32, _u8p, C.c_uint64)
        f("compact", C.c_void_p, C.POINTER(LoJob), C.POINTER(C.c_int))
        f("read_table", C.c_void_p, _u8p, C.c_uint64, C.POINTER(C.c_int))
        f("result_entries", C.c_uint64, C.c_void_p, C.c_int)
    else:
        f("crc32c", C.c_uint32, _u8p, C.c_uint64)
        f("compact", C.c_void_p, C.POINTER(RefJob))
        f("compact_parallel", C.c_double, C.POINTER(RefJob), C.c_int, C.POINTER(C.c_int))
        f("result_status", C.c_int, C.c_void_p)
        f("result_message", C.c_char_p, C.c_void_p)
        f("result_seconds", C.c_double, C.c_void_p)
        f("read_table", C.c_void_p, _u8p, C.c_uint64, C.c_int, C.POINTER(C.c_int))


def lib(impl: str = "oracle"):
    """The loaded checker library: ``"oracle"`` (restatement) or ``"ref"``."""
    if impl in _libs:
        return _libs[impl]
    path = ORACLE_SO if impl == "oracle" else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (make -C oracle{' ref' if impl == 'ref' else ''})")
    l = C.CDLL(path)
    _bind(l, "lo_" if impl == "oracle" else "ref_")
    _libs[impl] = (l, "lo_" if impl == "oracle" else "ref_")
    return _libs[impl]


def has_ref() -> bool:
    return os.path.exists(REF_SO)


# The reference LevelDB driven through leveldb::DB by oracle/db_scenario.cc:
# with the reference's CPU DoCompactionWork, and with the luda_b200 drop-in.
SCENARIO_CPU = os.path.join(HERE, "_ref", "db_scenario_cpu")
SCENARIO_DROPIN = os.path.join(HERE, "_ref", "db_scenario_luda_b200")


def run_scenario(exe: str, db_dir: str, seed: int, timeout_s: float = 300.0) -> dict:
    """Runs one scenario executable on a fresh DB directory; its JSON line."""
    import json
    r = subprocess.run([exe, db_dir, str(seed)], capture_output=True, text=True,
                       timeout=timeout_s)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed ({r.returncode}): "
                           f"{r.stdout[-500:]} {r.stderr[-500:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def _ptr(a: np.ndarray, t=_u8p):
    return a.ctypes.data_as(t)


def _call(impl, name):
    l, p = lib(impl)
    return getattr(l, p + name)


def _take_buf(impl, h) -> bytes:
    n = C.c_uint64()
    p = _call(impl, "buf_data")(h, C.byref(n))
    out = C.string_at(p, n.value) if n.value else b""
    _call(impl, "buf_free")(h)
    return out


def _u8(b) -> np.ndarray:
    if isinstance(b, np.ndarray):
        return np.ascontiguousarray(b, dtype=np.uint8)
    return np.frombuffer(bytes(b), np.uint8) if len(b) else np.zeros(1, np.uint8)


# -- primitives ------------------------------------------------------------

def crc32c(data: bytes, impl: str = "oracle") -> int:
    a = _u8(data)
    if impl == "oracle":
        return _call(impl, "crc32c_extend")(0, _ptr(a), len(data))
    return _call(impl, "crc32c")(_ptr(a), len(data))


def crc32c_mask(crc: int, impl: str = "oracle") -> int:
    return _call(impl, "crc32c_mask")(crc)


def leveldb_hash(data: bytes, seed: int, impl: str = "oracle") -> int:
    a = _u8(data)
    return _call(impl, "hash")(_ptr(a), len(data), seed)


def _pack_keys(keys: List[bytes]):
    offs = np.zeros(len(keys) + 1, np.uint64)
    offs[1:] = np.cumsum([len(k) for k in keys], dtype=np.uint64) if keys else []
    data = _u8(b"".join(keys))
    return data, offs


def bloom(keys: List[bytes], bits_per_key: int, impl: str = "oracle") -> bytes:
    data, offs = _pack_keys(keys)
    return _take_buf(impl, _call(impl, "bloom")(bits_per_key, len(keys), _ptr(data),
                                                _ptr(offs, _u64p)))


def separator(a: bytes, b: bytes, impl: str = "oracle") -> bytes:
    x, y = _u8(a), _u8(b)
    return _take_buf(impl, _call(impl, "separator")(_ptr(x), len(a), _ptr(y), len(b)))


def successor(a: bytes, impl: str = "oracle") -> bytes:
    x = _u8(a)
    return _take_buf(impl, _call(impl, "successor")(_ptr(x), len(a)))


# -- tables ----------------------------------------------------------------

def build_table(entries, options, impl: str = "oracle") -> bytes:
    """TableBuilder over ``luda_b200.job.Entries`` (sorted internal keys)."""
    keys = _u8(entries.keys)
    vals = _u8(entries.vals)
    ko = np.ascontiguousarray(entries.koffs, np.uint64)
    vo = np.ascontiguousarray(entries.voffs, np.uint64)
    h = _call(impl, "build_table")(options.block_size, options.restart_interval,
                                   options.bits_per_key, entries.n, _ptr(keys), _ptr(ko, _u64p),
                                   _ptr(vals), _ptr(vo, _u64p))
    return _take_buf(impl, h)


def read_table(data: bytes, impl: str = "oracle", bits_per_key: int = 10):
    """All (internal key, value) pairs of a table, or raises ValueError."""
    a = _u8(data)
    st = C.c_int()
    if impl == "oracle":
        h = _call(impl, "read_table")(_ptr(a), len(data), C.byref(st))
    else:
        h = _call(impl, "read_table")(_ptr(a), len(data), bits_per_key, C.byref(st))
    raw = _take_buf(impl, h)
    if st.value != 0:
        raise ValueError(f"table unreadable ({st.value}): {raw[:200]!r}")
    out = []
    pos = 0
    while pos < len(raw):
        kl = int.from_bytes(raw[pos:pos + 4], "little")
        k = raw[pos + 4:pos + 4 + kl]
        pos += 4 + kl
        vl = int.from_bytes(raw[pos:pos + 4], "little")
        v = raw[pos + 4:pos + 4 + vl]
        pos += 4 + vl
        out.append((k, v))
    return out


# -- compaction ------------------------------------------------------------

class _Keep:
    """Keeps numpy buffers alive while a ctypes struct points into them."""

    def __init__(self):
        self.objs = []

    def u8(self, b):
        a = _u8(b)
        self.objs.append(a)
        return _ptr(a)


def _lo_job(job, keep: _Keep) -> LoJob:
    runs = job.runs()
    tables = [f for r in runs for f in r]
    t_arr = (LoTable * max(1, len(tables)))()
    for i, f in enumerate(tables):
        t_arr[i].data = keep.u8(f.data)
        t_arr[i].size = len(f.data)
    rc = (C.c_int32 * max(1, len(runs)))(*[len(r) for r in runs])

    def ranges(fs):
        arr = (LoFileRange * max(1, len(fs)))()
        for i, f in enumerate(fs):
            arr[i].smallest = keep.u8(f.smallest)
            arr[i].smallest_len = len(f.smallest)
            arr[i].largest = keep.u8(f.largest)
            arr[i].largest_len = len(f.largest)
            arr[i].file_size = f.file_size
            arr[i].level = f.level
        return arr

    gp = job.grandparents()
    base = job.base_files()
    gpa, ba = ranges(gp), ranges(base)
    keep.objs += [t_arr, rc, gpa, ba]
    o = job.options
    return LoJob(job.level, len(tables), t_arr, len(runs), rc, len(gp), gpa, len(base), ba,
                 job.smallest_snapshot(), o.block_size, o.restart_interval, o.bits_per_key,
                 o.max_file_size)


def _ref_job(job, keep: _Keep) -> RefJob:
    files = job.files
    arr = (RefFile * max(1, len(files)))()
    for i, f in enumerate(files):
        if f.data is not None:
            arr[i].data = keep.u8(f.data)
        arr[i].size = f.file_size
        arr[i].level = f.level
        arr[i].smallest = keep.u8(f.smallest)
        arr[i].smallest_len = len(f.smallest)
        arr[i].largest = keep.u8(f.largest)
        arr[i].largest_len = len(f.largest)
    snaps = np.array(job.snapshots or [0], np.uint64)
    keep.objs += [arr, snaps]
    o = job.options
    return RefJob(job.level, len(files), arr, len(job.snapshots), _ptr(snaps, _u64p),
                  job.last_sequence, o.block_size, o.restart_interval, o.bits_per_key,
                  o.max_file_size)


def compact(job, impl: str = "oracle") -> List[Tuple[bytes, bytes, bytes]]:
    """Runs one compaction on a CPU checker.  Returns ``(file bytes,
    smallest internal key, largest internal key)`` per output file."""
    keep = _Keep()
    if impl == "oracle":
        j = _lo_job(job, keep)
        st = C.c_int()
        h = _call(impl, "compact")(C.byref(j), C.byref(st))
        status = st.value
    else:
        j = _ref_job(job, keep)
        h = _call(impl, "compact")(C.byref(j))
        status = _call(impl, "result_status")(h)
    try:
        if status != 0:
            msg = _call(impl, "result_message")(h).decode() if impl == "ref" else ""
            raise RuntimeError(f"{impl} compaction failed: status {status} {msg}")
        out = []
        for i in range(_call(impl, "result_nfiles")(h)):
            n = C.c_uint64()
            p = _call(impl, "result_file")(h, i, C.byref(n))
            data = C.string_at(p, n.value)
            m = C.c_uint32()
            p = _call(impl, "result_smallest")(h, i, C.byref(m))
            sm = C.string_at(p, m.value)
            p = _call(impl, "result_largest")(h, i, C.byref(m))
            lg = C.string_at(p, m.value)
            out.append((data, sm, lg))
        return out
    finally:
        _call(impl, "result_free")(h)


def ref_compact_timed(job) -> Tuple[List[Tuple[bytes, bytes, bytes]], float]:
    """The reference's DoCompactionWork; returns outputs and its wall seconds."""
    keep = _Keep()
    j = _ref_job(job, keep)
    h = _call("ref", "compact")(C.byref(j))
    try:
        status = _call("ref", "result_status")(h)
        if status != 0:
            raise RuntimeError(_call("ref", "result_message")(h).decode())
        secs = _call("ref", "result_seconds")(h)
        out = []
        for i in range(_call("ref", "result_nfiles")(h)):
            n = C.c_uint64()
            p = _call("ref", "result_file")(h, i, C.byref(n))
            out.append(C.string_at(p, n.value))
        return out, secs
    finally:
        _call("ref", "result_free")(h)


def ref_compact_parallel(job, n_threads: int) -> float:
    """Wall seconds for ``n_threads`` concurrent copies of the job on the
    reference CPU path (one DB each)."""
    keep = _Keep()
    j = _ref_job(job, keep)
    st = C.c_int()
    secs = _call("ref", "compact_parallel")(C.byref(j), n_threads, C.byref(st))
    if st.value != 0:
        raise RuntimeError("reference parallel compaction failed")
    return secs


def oracle_compact_timed(job) -> Tuple[List[Tuple[bytes, bytes, bytes]], float]:
    import time
    t0 = time.perf_counter()
    out = compact(job, "oracle")
    return out, time.perf_counter() - t0
