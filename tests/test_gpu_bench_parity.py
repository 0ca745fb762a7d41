"""Every configuration the benchmark times, compared with the oracle at full size.

* The 64-job batched workload at scale 1 (log-uniform 1-64 MiB per job, 2-12
  tables, 16-byte keys, 100-byte values; the seeds the benchmark's rank 0
  uses) through one lc_compact_batch call from host buffers: every output file
  of every job must equal the C restatement's, and for four of the jobs the
  reference's own CPU DoCompactionWork (oracle/_ref) when it is present.
* The served loop at the benchmark's scale (4 MiB level-0 flushes of 16-byte
  keys and 100-byte values, the default 2 MiB max_file_size, level sizes as
  LevelDB's): every job the loop ran must give the restatement's bytes.
"""
import os
import sys

import pytest

import oracle
from luda_b200 import served, workloads
from luda_b200.engine import Engine

sys.path.insert(0, os.path.dirname(__file__))
from test_served import _newest, db_contents  # noqa: E402

pytestmark = pytest.mark.gpu


def test_batched_64_full_size_matches_oracle(engine):
    jobs = [workloads.batched_job(s) for s in range(64)]
    for j in jobs:
        j.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    assert sum(j.input_bytes() for j in jobs) > 400 << 20
    res = engine.run_batch([engine.prepare(j) for j in jobs])
    for k, (j, r) in enumerate(zip(jobs, res)):
        want = oracle.compact(j, "oracle")
        assert r.file_bytes() == [w[0] for w in want], j.name
        assert [(f.smallest, f.largest) for f in r.files] == [(w[1], w[2]) for w in want], j.name
        if k % 16 == 0 and oracle.has_ref():
            assert [w[0] for w in oracle.compact(j, "ref")] == [w[0] for w in want], j.name
        r.release()


def test_served_bench_scale_matches_oracle(engine):
    from luda_b200.device_buffers import TorchUploader
    fl = served.make_flushes(4, 16, lambda e, o: engine.build_table(e, o), seed=3)
    assert all(len(f.data) > 3 << 20 for f in fl[0])
    up = TorchUploader(0)
    with Engine(0, max_inflight=4) as eng:
        srv = served.Server(eng, len(fl), mode="served", upload=up.upload, free=up.free,
                            ready=up.ready, record_bytes=True)
        st = srv.run(served.schedule(fl, None))
        assert {j.level for j in st.jobs} >= {0, 1}
        assert any(j.resident_inputs == j.n_inputs and j.n_inputs > 0 for j in st.jobs)
        # outputs of earlier jobs are read from their decoded form
        assert any(j.decoded_inputs > 0 for j in st.jobs)
        for rec in st.jobs:
            assert [o[0] for o in oracle.compact(rec.job, "oracle")] == rec.file_bytes
        for db, f in zip(srv.dbs, fl):
            db.check_levels()
            assert db_contents(db) == _newest([f])
        srv.close()
