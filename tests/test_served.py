"""The served request loop's host logic, on the CPU.

The loop drives several simulated databases through a fake engine whose
compactions are the oracle's (the CPU restatement), with completions in a
shuffled order.  After the run every database must hold exactly the newest
value of every key written, in levels whose key ranges are disjoint and
ordered, and the loop must have run compactions at several levels.
"""
import numpy as np
import pytest

import oracle
from luda_b200 import served
from luda_b200.job import TableOptions


class _Res:
    def __init__(self, outs):
        self.files = [type("F", (), {"data": memoryview(d), "smallest": s, "largest": l})
                      for d, s, l in outs]
        self.bytes_out = sum(len(d) for d, _, _ in outs)
        self.device_ptr = None
        self.file_offsets = None
        self.released = False

    def release(self):
        assert not self.released
        self.released = True

    def file_bytes(self):
        return [bytes(f.data) for f in self.files]


class _Async:
    def __init__(self, res):
        self.res, self.h = res, object()

    def wait(self):
        return self.res


class OracleEngine:
    """prepare / submit_prepared / wait_any over oracle.compact."""

    def __init__(self, seed=0):
        self.rng = np.random.default_rng(seed)
        self.jobs = 0

    def prepare(self, job, device_tables=None, outputs_on_device=0, keep_decoded=False,
                decoded=None):
        # the real engine takes the table pointers here; the host may drop
        # its references to the job's buffers right after
        assert device_tables is None
        for f in job.input_tables():
            assert f.data is not None and len(f.data) == f.file_size
        return oracle.compact(job, "oracle")

    def submit_prepared(self, outs):
        self.jobs += 1
        return _Async(_Res(outs))

    def wait_any(self, jobs, timeout_s=-1.0):
        return int(self.rng.integers(0, len(jobs)))


def _newest(flushes):
    """user key -> value bytes of its newest put, over every flush."""
    want = {}
    for fl in flushes:
        for f in fl:
            for k, v in oracle.read_table(bytes(f.data)):
                seq = int.from_bytes(k[-8:], "little") >> 8
                uk = k[:-8]
                if uk not in want or want[uk][0] < seq:
                    want[uk] = (seq, v)
    return {k: v for k, (s, v) in want.items()}


def db_contents(db):
    """user key -> value, reading newest tables first (level 0 newest file
    first, then each deeper level)."""
    got = {}
    tables = list(reversed(db.levels[0])) + [t for lvl in db.levels[1:] for t in lvl]
    for t in tables:
        for k, v in oracle.read_table(bytes(t.host)):
            got.setdefault(k[:-8], v)
    return got


@pytest.fixture(scope="module")
def small_flushes(oracle_lib):
    opts = TableOptions(max_file_size=64 << 10)
    return opts, served.make_flushes(3, 14, lambda e, o: oracle.build_table(e, o, "oracle"),
                                     seed=5, options=opts, entries_per_flush=1500)


@pytest.mark.parametrize("mode", ["plain", "served"])
def test_served_loop_keeps_newest_values(small_flushes, mode):
    opts, flushes = small_flushes
    eng = OracleEngine(seed=1)
    srv = served.Server(eng, len(flushes), mode=mode, options=opts, level_scale=1 / 128.0)
    st = srv.run(served.schedule(flushes, None), idle_wait=lambda s: None)
    levels_used = set()
    for db, fl in zip(srv.dbs, flushes):
        db.check_levels()
        levels_used |= {lvl for lvl, ts in enumerate(db.levels) if ts and lvl > 0}
        assert db_contents(db) == _newest([fl])
    assert st.flushes == sum(len(f) for f in flushes)
    assert {1, 2} <= levels_used
    assert len(st.jobs) == eng.jobs and eng.jobs > 0
    assert {j.level for j in st.jobs} >= {0, 1}
    s = st.summary()
    assert s["jobs"] == len(st.jobs) and s["p99_ms"] >= s["p50_ms"]
    srv.close()


def test_uploads_ready_before_a_job_reads_them(small_flushes):
    """Level-0 uploads may still be in flight when upload() returns: the loop
    must call ready() on every uploaded table before it hands the table's
    device address to a job."""
    opts, flushes = small_flushes
    handles = {}

    def upload(data):
        addr = 4096 * (len(handles) + 1)
        handles[addr] = {"ready": False}
        return addr, handles[addr]

    def ready(h):
        h["ready"] = True

    class DeviceOracle(OracleEngine):
        device_jobs = 0

        def prepare(self, job, device_tables=None, outputs_on_device=0, keep_decoded=False,
                decoded=None):
            if device_tables is not None:
                assert all(handles[a]["ready"] for a in device_tables)
                self.device_jobs += 1
            for f in job.input_tables():
                f.data = f.sim.host
            return oracle.compact(job, "oracle")

    eng = DeviceOracle(seed=2)
    srv = served.Server(eng, len(flushes), mode="served", options=opts, upload=upload,
                        free=lambda h: None, ready=ready, level_scale=1 / 128.0)
    srv.run(served.schedule(flushes, None), idle_wait=lambda s: None)
    assert eng.device_jobs > 0
    for db, fl in zip(srv.dbs, flushes):
        assert db_contents(db) == _newest([fl])
    srv.close()


def test_pick_follows_compaction_pointer():
    db = served.SimDB(0, TableOptions(), level_scale=1e-6)

    def t(n, a, b, lvl=1):
        return served.SimTable(n, lvl, a.encode() + b"\x01" * 8, b.encode() + b"\x01" * 8, 10)
    db.levels[1] = [t(1, "a", "c"), t(2, "d", "f"), t(3, "g", "i")]
    db.levels[2] = [t(4, "b", "e", 2), t(5, "h", "z", 2)]
    lvl, in0, in1, gp = db.pick()
    assert lvl == 1 and [f.number for f in in0] == [1] and [f.number for f in in1] == [4]
    lvl, in0, in1, gp = db.pick()
    assert [f.number for f in in0] == [2] and [f.number for f in in1] == [4]
    lvl, in0, in1, gp = db.pick()
    assert [f.number for f in in0] == [3] and [f.number for f in in1] == [5]
    lvl, in0, in1, gp = db.pick()  # wraps around
    assert [f.number for f in in0] == [1]


def test_level0_overlap_widens():
    db = served.SimDB(0, TableOptions())

    def t(n, a, b):
        return served.SimTable(n, 0, a.encode() + b"\x01" * 8, b.encode() + b"\x01" * 8, 10)
    db.levels[0] = [t(1, "m", "p"), t(2, "a", "n"), t(3, "o", "z"), t(4, "q", "r")]
    got = db.overlapping(0, db.levels[0][0].smallest, db.levels[0][0].largest)
    assert sorted(f.number for f in got) == [1, 2, 3, 4]


def test_schedule_poisson_rate():
    fl = [[served.Flush(0.0, d, b"", b"", b"", 0) for _ in range(200)] for d in range(5)]
    arr = served.schedule(fl, 1000.0, seed=2)
    assert len(arr) == 1000
    ts = np.array([a.t for a in arr])
    assert np.all(np.diff(ts) >= 0)
    assert 0.8 < ts[-1] < 1.2  # 1000 arrivals at 1000/s
    assert sorted(a.db for a in arr) == sorted(d for d in range(5) for _ in range(200))
