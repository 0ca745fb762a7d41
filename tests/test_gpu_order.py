"""Inputs whose entries are out of internal-key order.

A table's blocks can be intact (valid trailers and CRCs) while its entries
are not sorted: a buggy writer, or a table built from unsorted input.  The
reference merges its children trusting their order (table/merger.cc), and the
merge path here cuts the output by binary searches that assume it.  The engine
checks every child's order on the device before the merge and fails such a
job with a corruption status naming the order; the other jobs of a batch and
the engine itself are unaffected.
"""
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.engine import LcError
from luda_b200.job import Entries

pytestmark = pytest.mark.gpu


def _job(seed, swap=None, common_prefix=False):
    job = workloads.plain_l0_l1(seed=seed, scale=0.02)
    if swap is not None:
        f = next(f for f in job.files if f.entries is not None and f.entries.n > 100)
        e = f.entries
        keys = [e.key(i) for i in range(e.n)]
        vals = [e.value(i) for i in range(e.n)]
        i, j = swap(e.n)
        keys[i], keys[j] = keys[j], keys[i]
        vals[i], vals[j] = vals[j], vals[i]
        f.entries = Entries.from_lists(keys, vals)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    return job


@pytest.mark.parametrize("swap", [lambda n: (0, 1), lambda n: (n // 3, n // 2),
                                  lambda n: (n - 2, n - 1)],
                         ids=["head", "middle", "tail"])
def test_out_of_order_child_fails(engine, swap):
    bad = _job(21, swap)
    with pytest.raises(LcError) as ei:
        engine.compact(bad)
    assert ei.value.status == 2 and "order" in str(ei.value)
    ok = _job(22)
    assert engine.compact(ok).file_bytes() == [x[0] for x in oracle.compact(ok, "oracle")]


def test_out_of_order_stays_in_its_job(engine):
    good = [_job(s) for s in (23, 24)]
    bad = _job(25, lambda n: (n // 4, 3 * n // 4))
    res = engine.run_batch([engine.prepare(good[0]), engine.prepare(bad), engine.prepare(good[1])],
                           errors="return")
    assert isinstance(res[1], LcError) and res[1].status == 2 and "order" in str(res[1])
    for r, j in ((res[0], good[0]), (res[2], good[1])):
        assert r.file_bytes() == [x[0] for x in oracle.compact(j, "oracle")]
