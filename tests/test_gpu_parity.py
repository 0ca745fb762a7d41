"""Parity of the GPU engine with the reference, through the C ABI.

Byte identity is the bar: every output file of every fixture case must have
the SHA-256, size and smallest/largest internal keys that the reference's CPU
DoCompactionWork produced (tests/golden/golden.json), and must equal the CPU
restatement's output on the same inputs.  Inputs are rebuilt from the seeded
generators; their hashes are checked against the fixture first.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.job import Entries, TableOptions

sys.path.insert(0, os.path.dirname(__file__))
from test_oracle import golden_job, _golden  # noqa: E402

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(b).hexdigest()


ALL = [c for c in _golden() if not c.get("large")]  # 1 GiB cases: test_gpu_large.py


@pytest.fixture(scope="module")
def built_jobs(oracle_lib):
    cache = {}

    def get(case):
        if case["name"] not in cache:
            job = golden_job(case)
            job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
            assert [sha(f.data) for f in job.input_tables()] == case["inputs"]
            cache[case["name"]] = job
        return cache[case["name"]]
    return get


@pytest.mark.parametrize("case", ALL, ids=[c["name"] for c in ALL])
def test_compaction_matches_reference(engine, built_jobs, case):
    job = built_jobs(case)
    res = engine.compact(job)
    assert len(res.files) == len(case["outputs"])
    for f, g in zip(res.files, case["outputs"]):
        assert len(f.data) == g["size"]
        assert sha(bytes(f.data)) == g["sha256"]
        assert f.smallest.hex() == g["smallest"]
        assert f.largest.hex() == g["largest"]
    assert res.bytes_in == case["input_bytes"]


@pytest.mark.parametrize("case", [c for c in ALL if c["input_bytes"] < 8 << 20][:12],
                         ids=lambda c: c["name"])
def test_compaction_matches_oracle(engine, built_jobs, case):
    job = built_jobs(case)
    res = engine.compact(job)
    ref = oracle.compact(job, "oracle")
    assert res.file_bytes() == [r[0] for r in ref]
    assert [f.entries for f in res.files] == [len(oracle.read_table(r[0])) for r in ref]


@pytest.mark.parametrize("bs,ri,bpk", [(4096, 16, 10), (1024, 1, 0), (65536, 3, 20),
                                       (2048, 16, 1)])
def test_flush_encoder_matches_table_builder(engine, bs, ri, bpk):
    job = workloads.plain_l0_l1(seed=5, scale=0.2)
    opts = TableOptions(block_size=bs, restart_interval=ri, bits_per_key=bpk)
    for f in job.files:
        got = engine.build_table(f.entries, opts)
        want = oracle.build_table(f.entries, opts, "oracle")
        assert got == want


def test_flush_encoder_variable_keys(engine):
    job = workloads.l1_l2_at_size(seed=3, scale=0.05, n_l2_tables=4, n_l3_files=4)
    for f in job.files:
        if f.entries is not None:
            assert engine.build_table(f.entries, job.options) == \
                oracle.build_table(f.entries, job.options, "oracle")


def test_outputs_readable(engine, built_jobs):
    case = [c for c in ALL if c["name"] == "snapshot_versions"][0]
    job = built_jobs(case)
    res = engine.compact(job)
    for f in res.files:
        ents = oracle.read_table(bytes(f.data))
        assert len(ents) == f.entries
        assert ents[0][0] == f.smallest and ents[-1][0] == f.largest
        if oracle.has_ref():
            assert oracle.read_table(bytes(f.data), "ref") == ents


def test_device_resident_equals_host(engine, built_jobs):
    import torch
    case = [c for c in ALL if c["name"] == "plain_l0_l1"][0]
    job = built_jobs(case)
    host = engine.compact(job)
    tables = job.input_tables()
    offs, total = [], 0
    for f in tables:
        offs.append(total)
        total += (len(f.data) + 15) // 16 * 16
    buf = torch.zeros(total + 16, dtype=torch.uint8, device="cuda")
    for f, o in zip(tables, offs):
        buf[o:o + len(f.data)] = torch.frombuffer(bytearray(f.data), dtype=torch.uint8).cuda()
    torch.cuda.synchronize()
    dev = engine.compact(job, device_tables=[buf.data_ptr() + o for o in offs],
                         outputs_on_device=True)
    assert len(dev.files) == len(host.files)
    from cuda.bindings import runtime as rt
    for i, f in enumerate(host.files):
        size = len(f.data)
        host_buf = np.empty(size, np.uint8)
        err, = rt.cudaMemcpy(host_buf.ctypes.data, dev.device_ptr + dev.file_offsets[i], size,
                             rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        assert host_buf.tobytes() == bytes(f.data)


def test_async_jobs_same_alone_and_in_mix(engine, built_jobs):
    names = ["batched_0", "batched_1", "batched_2", "batched_3", "plain_l0_l1_small",
             "many_files"]
    cases = [c for c in ALL if c["name"] in names]
    jobs = [built_jobs(c) for c in cases]
    alone = [engine.compact(j) for j in jobs]
    handles = [engine.submit(j) for j in jobs * 2]
    mixed = [h.wait() for h in handles]
    for a, m in zip(alone * 2, mixed):
        assert a.file_bytes() == m.file_bytes()


def _corrupt(job, fn):
    t = job.input_tables()[0]
    b = bytearray(t.data)
    fn(b)
    t.data = bytes(b)
    return job


@pytest.mark.parametrize("kind", ["magic", "index_handle", "restart_count", "truncated"])
def test_corrupt_input_reports_corruption(engine, kind):
    from luda_b200.engine import LcError
    job = workloads.plain_l0_l1(seed=8, scale=0.02)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))

    def f(b):
        if kind == "magic":
            b[-1] ^= 0xFF
        elif kind == "index_handle":
            b[-48] = 0xFF
            b[-47] = 0xFF
            b[-46] = 0xFF
            b[-45] = 0x7F
        elif kind == "restart_count":
            # first data block: make its restart count huge
            n = len(b)
            foot = b[n - 48:]
            b[0:4] = b"\x7f\x7f\x7f\x7f"
        elif kind == "truncated":
            del b[len(b) // 2:len(b) // 2 + 100]
    _corrupt(job, f)
    with pytest.raises(LcError) as ei:
        engine.compact(job)
    assert ei.value.status in (2, 7)
    # the engine stays usable
    ok = workloads.plain_l0_l1(seed=8, scale=0.02)
    ok.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    assert engine.compact(ok).file_bytes() == [x[0] for x in oracle.compact(ok)]


def test_shared_prefix_keys_rerun_with_counting(engine):
    """Keys that share 200 bytes with their predecessor decode to about ten
    times the table bytes: the single-pass key arena (the input size) is too
    small, the engine reruns the job with exact counting, and the output is
    still the reference's."""
    from luda_b200.job import CompactionJob, FileMeta, internal_key
    prefix = b"p" * 200
    opts = TableOptions(max_file_size=1 << 20)

    def table(number, ids, seq0):
        keys = [internal_key(prefix + b"%012d" % i, seq0 + k, 1) for k, i in enumerate(ids)]
        e = Entries.from_lists(keys, [b""] * len(keys))
        return FileMeta(number == 1 and 0 or 1, number, keys[0], keys[-1], 0, e, None)
    files = [table(1, range(0, 20000, 2), 100000), table(2, range(0, 20000, 3), 1)]
    files[0].level = 0
    files[1].level = 1
    job = CompactionJob(0, files, [], 200000, opts, name="shared_prefix")
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    assert sum(f.entries.n for f in files) * 212 > 2 * job.input_bytes()
    res = engine.compact(job)
    assert res.file_bytes() == [r[0] for r in oracle.compact(job, "oracle")]
