"""Served compaction on the GPU: every job's result is the same alone and in
the mix.

Several simulated databases run their compactions through one engine with
continuous batching, device-resident level-0 uploads and outputs kept on the
device, with their decoded entries, for the next level's jobs (which then read
those inputs without parsing or decoding them).  Each job the loop ran is then compacted
again alone from host copies of its inputs (lc_compact) and by the CPU
restatement; all three must be byte-identical, and every database must end up
holding the newest value of every key written.
"""
import os
import sys

import pytest

import oracle
from luda_b200 import served
from luda_b200.engine import Engine
from luda_b200.job import TableOptions

sys.path.insert(0, os.path.dirname(__file__))
from test_served import _newest, db_contents  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def flushes(engine):
    opts = TableOptions(max_file_size=256 << 10)
    return opts, served.make_flushes(4, 12, lambda e, o: engine.build_table(e, o), seed=9,
                                     options=opts, entries_per_flush=4000)


@pytest.mark.parametrize("rate", [None, 400.0])
def test_served_jobs_same_alone_and_in_mix(flushes, rate):
    from luda_b200.device_buffers import TorchUploader
    opts, fl = flushes
    up = TorchUploader(0)
    with Engine(0, max_inflight=3) as eng:
        srv = served.Server(eng, len(fl), mode="served", options=opts, upload=up.upload,
                            free=up.free, ready=up.ready, record_bytes=True,
                            level_scale=1 / 16.0)
        st = srv.run(served.schedule(fl, rate))
        assert len(st.jobs) > 0 and {j.level for j in st.jobs} >= {0, 1}
        assert any(j.resident_inputs == j.n_inputs and j.n_inputs > 0 for j in st.jobs)
        # outputs of earlier jobs are read from their decoded form
        assert any(j.decoded_inputs > 0 for j in st.jobs)
        for rec in st.jobs:
            alone = eng.compact(rec.job)
            assert alone.file_bytes() == rec.file_bytes
            alone.release()
            assert [o[0] for o in oracle.compact(rec.job, "oracle")] == rec.file_bytes
        for db, f in zip(srv.dbs, fl):
            db.check_levels()
            assert db_contents(db) == _newest([f])
        srv.close()


def test_plain_mode_same_bytes(flushes):
    opts, fl = flushes
    with Engine(0, max_inflight=1, max_batch=1) as eng:
        srv = served.Server(eng, len(fl), mode="plain", options=opts, record_bytes=True,
                            level_scale=1 / 16.0)
        st = srv.run(served.schedule(fl, None))
        for rec in st.jobs[:10]:
            assert [o[0] for o in oracle.compact(rec.job, "oracle")] == rec.file_bytes
        srv.close()


def test_wait_any_and_outputs_both(flushes):
    """lc_job_wait_any returns finished jobs; outputs_on_device=2 gives the
    same bytes in host and device memory."""
    import numpy as np
    import torch
    from luda_b200 import workloads
    jobs = [workloads.batched_job(s, scale=0.02) for s in range(4)]
    for j in jobs:
        j.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    with Engine(0, max_inflight=2) as eng:
        hs = [eng.submit_prepared(eng.prepare(j, outputs_on_device=2)) for j in jobs]
        seen = set()
        while len(seen) < len(hs):
            live = [i for i in range(len(hs)) if i not in seen]
            k = eng.wait_any([hs[i] for i in live], 30.0)
            assert k is not None
            seen.add(live[k])
        for h, j in zip(hs, jobs):
            r = h.wait()
            want = [o[0] for o in oracle.compact(j, "oracle")]
            assert r.file_bytes() == want
            assert r.device_ptr
            for i, f in enumerate(r.files):
                n = len(f.data)
                buf = torch.empty(n, dtype=torch.uint8)
                from cuda.bindings import runtime as rt
                err, = rt.cudaMemcpy(buf.data_ptr(), r.device_ptr + r.file_offsets[i], n,
                                     rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
                assert err == rt.cudaError_t.cudaSuccess
                assert buf.numpy().tobytes() == want[i]
            r.release()
        st = eng.stats()
        assert st["jobs"] == 4 and st["queued_jobs"] == 0
