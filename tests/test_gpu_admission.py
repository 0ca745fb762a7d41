"""Admission against the device budget, and the waits' timeouts.

* A job whose admission estimate (lc_estimate_device_bytes) exceeds the
  engine's device budget is refused at submit with LC_ERR_BUDGET.
* With a budget that holds one job but not two, the second of two jobs
  submitted together waits in the queue until the first has finished (two
  workers are idle, so without the budget both would start at once).
* lc_job_wait and lc_job_wait_any return LC_ERR_TIMEOUT when the job is not
  done within the timeout; the job still completes and gives its bytes.
"""
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.engine import Engine, LcError

pytestmark = pytest.mark.gpu

LC_ERR_BUDGET = 5


@pytest.fixture(scope="module")
def job_pair(engine):
    jobs = [workloads.batched_job(s, scale=1.0) for s in (4, 3)]  # 29 and 16 MiB
    for j in jobs:
        j.materialize(lambda e, o: engine.build_table(e, o))
    return jobs


def test_over_budget_job_is_refused(job_pair):
    with Engine(0, budget_bytes=16 << 20) as eng:
        p = eng.prepare(job_pair[0])
        assert eng.estimate_device_bytes(p) > 16 << 20
        with pytest.raises(LcError) as ex:
            eng.submit_prepared(p)
        assert ex.value.status == LC_ERR_BUDGET


def test_budget_holds_second_job_until_first_finishes(job_pair):
    big = max(job_pair, key=lambda j: j.input_bytes())
    small = min(job_pair, key=lambda j: j.input_bytes())
    with Engine(0) as probe:
        e_big = probe.estimate_device_bytes(probe.prepare(big))
        e_small = probe.estimate_device_bytes(probe.prepare(small))
    budget = max(e_big, e_small) + min(e_big, e_small) // 4
    with Engine(0, budget_bytes=budget, max_inflight=2) as eng:
        # warm the engine (slabs, pinned memory) so that timing is the jobs'
        eng.run(eng.prepare(small)).release()
        h1 = eng.submit_prepared(eng.prepare(big))
        h2 = eng.submit_prepared(eng.prepare(small))
        r1, r2 = h1.wait(), h2.wait()
        # the second job's batch started only after the first's had ended
        assert r2.queue_ms >= 0.8 * r1.device_ms, (r2.queue_ms, r1.device_ms)
        assert r1.batch_jobs == 1 and r2.batch_jobs == 1
        want = [o[0] for o in oracle.compact(small, "oracle")]
        assert r2.file_bytes() == want
        r1.release()
        r2.release()


def test_wait_and_wait_any_time_out(job_pair):
    job = max(job_pair, key=lambda j: j.input_bytes())
    with Engine(0, max_inflight=1) as eng:
        p = eng.prepare(job)
        eng.run(p).release()
        h = eng.submit_prepared(p)
        # a compaction of tens of MiB cannot be done within zero nanoseconds
        assert eng.wait_any([h], 0.0) is None
        with pytest.raises(TimeoutError):
            h.wait(0.0)
        r = h.wait()
        assert r.file_bytes() == [o[0] for o in oracle.compact(job, "oracle")]
        r.release()
