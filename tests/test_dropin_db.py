"""The compiled drop-in inside a real leveldb::DB.

oracle/Makefile (target dropin) builds the reference's LevelDB twice from the
reference sources: once with its own CPU DBImpl::DoCompactionWork
(db_scenario_cpu) and once with DoCompactionWork replaced by
luda_b200/host/do_compaction_work.cc, which runs the compaction through the
engine's C ABI (db_scenario_luda_b200).  Both run the same seeded scenario
through the public DB API (oracle/db_scenario.cc): writes, memtable flushes,
a snapshot, manual level-0 -> level-1 and level-1 -> level-2 compactions
(DBImpl::TEST_CompactRange), then reads everything back.

On the CPU (here) the reference twin must read back its model.  On the GPU
the drop-in must: every table file the two builds leave in their DB
directories has the same number and the same bytes, the DB reads back its
model through an iterator, Get and the snapshot, and the compactions ran
through the engine and were installed (InstallCompactionResults) -- the
levels the DB reports match.
"""
import os

import pytest

import oracle

needs_builds = pytest.mark.skipif(
    not (os.path.exists(oracle.SCENARIO_CPU) and os.path.exists(oracle.SCENARIO_DROPIN)),
    reason="drop-in scenario executables not built (oracle/Makefile dropin)")


def _tables(d):
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))
            if f.endswith(".ldb")}


@needs_builds
def test_reference_twin_reads_back_its_model(tmp_path):
    r = oracle.run_scenario(oracle.SCENARIO_CPU, str(tmp_path / "cpu"), 7)
    assert r["ok"] and r["mismatches"] == 0 and r["get_mismatches"] == 0
    assert r["snapshot_mismatches"] == 0 and r["entries"] == r["model_entries"] > 0
    assert r["served"] == -1
    assert sum(r["levels"]) > 0


@needs_builds
@pytest.mark.gpu
@pytest.mark.parametrize("seed", [7, 21])
def test_dropin_db_matches_reference_build(tmp_path, seed):
    cpu_dir, gpu_dir = str(tmp_path / "cpu"), str(tmp_path / "gpu")
    want = oracle.run_scenario(oracle.SCENARIO_CPU, cpu_dir, seed)
    got = oracle.run_scenario(oracle.SCENARIO_DROPIN, gpu_dir, seed)
    assert got["ok"], got
    assert got["mismatches"] == 0 and got["get_mismatches"] == 0
    assert got["snapshot_mismatches"] == 0
    assert got["entries"] == want["entries"] and got["levels"] == want["levels"]
    # three compactions of the scenario ran through the engine and were installed
    assert got["served"] >= 3
    a, b = _tables(cpu_dir), _tables(gpu_dir)
    assert sorted(a) == sorted(b)
    for name in a:
        assert a[name] == b[name], name
