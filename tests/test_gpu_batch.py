"""Batched compaction (lc_compact_batch), its CUDA graphs and the autotuner.

Every job of a batch must produce exactly the bytes it produces alone, which
the golden fixtures pin to the reference's CPU DoCompactionWork: uneven job
sizes, edge cases and failing jobs share the launches of one batch, graphs
captured for one batch are replayed for others, and every launch setting the
autotuner may pick gives the same output.
"""
import hashlib
import os
import sys

import pytest

import oracle
from luda_b200 import workloads
from luda_b200.engine import Engine, LcError

sys.path.insert(0, os.path.dirname(__file__))
from test_oracle import golden_job, _golden  # noqa: E402

pytestmark = pytest.mark.gpu

ALL = _golden()
SMALL = [c for c in ALL if c["input_bytes"] < 24 << 20]


def sha(b):
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="module")
def jobs_of(oracle_lib):
    cache = {}

    def get(case):
        if case["name"] not in cache:
            job = golden_job(case)
            job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
            cache[case["name"]] = job
        return cache[case["name"]]
    return get


def check_golden(res, case):
    assert len(res.files) == len(case["outputs"]), case["name"]
    for f, g in zip(res.files, case["outputs"]):
        assert sha(bytes(f.data)) == g["sha256"], case["name"]
        assert f.smallest.hex() == g["smallest"] and f.largest.hex() == g["largest"]


@pytest.fixture(scope="module")
def mix_jobs():
    jobs = [workloads.batched_job(s, scale=0.04) for s in range(12)]
    for j in jobs:
        j.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    return jobs


@pytest.fixture(scope="module")
def mix_want(mix_jobs):
    return [[x[0] for x in oracle.compact(j, "oracle")] for j in mix_jobs]


def test_batch_of_golden_cases(engine, jobs_of):
    res = engine.run_batch([engine.prepare(jobs_of(c)) for c in SMALL])
    for r, c in zip(res, SMALL):
        check_golden(r, c)
        assert r.bytes_in == c["input_bytes"]


def test_batch_uneven_jobs_match_oracle(engine, mix_jobs, mix_want):
    res = engine.compact_batch(mix_jobs)
    assert [r.file_bytes() for r in res] == mix_want


def test_graph_replay_for_other_batches(mix_jobs, mix_want):
    with Engine(0) as e:
        first = e.compact_batch(mix_jobs[:6])  # new shape: direct launches
        again = e.compact_batch(mix_jobs[:6])  # second sighting: captured
        third = e.compact_batch(mix_jobs[:6])  # replayed
        other = e.compact_batch(mix_jobs[6:])
        st = e.stats()
        assert st["direct_tails"] >= 1 and st["graph_captures"] >= 1 and st["graph_replays"] >= 1
        assert st["batches"] == 4 and st["jobs"] == 24
        for rs in (first, again, third):
            assert [r.file_bytes() for r in rs] == mix_want[:6]
        assert [r.file_bytes() for r in other] == mix_want[6:]


def test_no_graphs_same_bytes(mix_jobs, mix_want):
    with Engine(0, graphs=False) as e:
        assert [r.file_bytes() for r in e.compact_batch(mix_jobs)] == mix_want


def test_batches_split_at_max_batch(mix_jobs, mix_want):
    with Engine(0, max_batch=5) as e:
        assert [r.file_bytes() for r in e.compact_batch(mix_jobs)] == mix_want


def test_failed_job_does_not_disturb_batch(engine, mix_jobs, mix_want):
    bad = workloads.plain_l0_l1(seed=8, scale=0.02)
    bad.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    t = bad.input_tables()[0]
    b = bytearray(t.data)
    b[-1] ^= 0xFF  # table magic
    t.data = bytes(b)
    ps = [engine.prepare(j) for j in mix_jobs[:3]] + [engine.prepare(bad)] + \
        [engine.prepare(j) for j in mix_jobs[3:6]]
    res = engine.run_batch(ps, errors="return")
    assert isinstance(res[3], LcError) and res[3].status == 2
    good = res[:3] + res[4:]
    assert [r.file_bytes() for r in good] == mix_want[:6]
    with pytest.raises(LcError):
        engine.run_batch(ps)


@pytest.mark.parametrize("tun", [dict(ctas_per_job=1, merge_items=1, merge_threads=64),
                                 dict(ctas_per_job=3, merge_items=32, merge_threads=1024),
                                 dict(ctas_per_job=0, merge_items=5, merge_threads=96)])
def test_every_tuning_same_bytes(mix_jobs, mix_want, tun):
    with Engine(0) as e:
        e.set_tuning(**tun)
        assert e.tuning() == tun
        assert [r.file_bytes() for r in e.compact_batch(mix_jobs)] == mix_want


def test_autotune_picks_candidate_and_keeps_bytes(mix_jobs, mix_want):
    with Engine(0) as e:
        ps = [e.prepare(j) for j in mix_jobs]
        t = e.autotune(ps, repeats=1)
        assert t == e.tuning()
        assert t["merge_threads"] in (128, 256, 512) and t["merge_items"] in (4, 8, 16)
        assert [r.file_bytes() for r in e.run_batch(ps)] == mix_want


def test_bad_tuning_rejected(engine):
    with pytest.raises(LcError):
        engine.set_tuning(merge_items=0)
    with pytest.raises(LcError):
        engine.set_tuning(merge_threads=100)


def test_continuous_batching_same_alone_and_in_mix(mix_jobs, mix_want):
    # one worker: jobs queued while a batch runs join the next batch
    with Engine(0, max_inflight=1) as e:
        hs = [e.submit(j) for j in mix_jobs * 2]
        got = [h.wait().file_bytes() for h in hs]
    assert got == mix_want * 2


def test_large_host_batch_split_across_slots(engine):
    """Host inputs beyond 128 MiB in one lc_compact_batch call run as several
    parts on several streams at once; every job still gives the bytes it
    gives alone."""
    jobs = [workloads.batched_job(s) for s in range(40, 63)]
    for j in jobs:
        j.materialize(lambda e, o: engine.build_table(e, o))
    assert sum(j.input_bytes() for j in jobs) > 200 << 20
    ps = [engine.prepare(j) for j in jobs]
    alone = []
    for p in ps:
        r = engine.run(p)
        alone.append(r.file_bytes())
        r.release()
    before = engine.stats()["batches"]
    res = engine.run_batch(ps)
    assert engine.stats()["batches"] - before >= 3
    assert [r.file_bytes() for r in res] == alone
    for r in res:
        r.release()
