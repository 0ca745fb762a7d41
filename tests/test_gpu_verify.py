"""Device-side checksum verification of input blocks (verify_checksums).

LevelDB checks a block's CRC32C trailer on read when ReadOptions::
verify_checksums is set (table/format.cc:86-95); a compaction's inputs get it
from Options::paranoid_checks (db/version_set.cc:1239), and the reference
build has the check switched off.  With the option on, intact inputs compact
to the same bytes, and one flipped byte anywhere in the data blocks fails the
job with a corruption status that names the checksum -- without disturbing
the other jobs of a batch.
"""
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.engine import LcError

pytestmark = pytest.mark.gpu


def _job(seed=8):
    job = workloads.plain_l0_l1(seed=seed, scale=0.02)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    return job


def _flip(job, where):
    t = job.input_tables()[0]
    b = bytearray(t.data)
    b[where(len(b))] ^= 0x5A
    t.data = bytes(b)
    return job


def test_verified_compaction_same_bytes(engine):
    job = _job()
    want = [x[0] for x in oracle.compact(job, "oracle")]
    assert engine.compact(job, verify_checksums=True).file_bytes() == want
    assert engine.compact(job).file_bytes() == want


@pytest.mark.parametrize("where", [lambda n: 40, lambda n: n // 3, lambda n: n // 2],
                         ids=["first_block", "third", "middle"])
def test_flipped_byte_fails_checksum(engine, where):
    job = _flip(_job(), where)
    with pytest.raises(LcError) as ei:
        engine.compact(job, verify_checksums=True)
    assert ei.value.status == 2 and "checksum" in str(ei.value)
    # the engine stays usable
    ok = _job(seed=9)
    assert engine.compact(ok, verify_checksums=True).file_bytes() == \
        [x[0] for x in oracle.compact(ok, "oracle")]


def test_checksum_failure_stays_in_its_job(engine):
    good = [_job(seed=s) for s in (10, 11)]
    bad = _flip(_job(seed=12), lambda n: n // 3)
    ps = [engine.prepare(good[0], verify_checksums=True), engine.prepare(bad, verify_checksums=True),
          engine.prepare(good[1], verify_checksums=True)]
    res = engine.run_batch(ps, errors="return")
    assert isinstance(res[1], LcError) and res[1].status == 2 and "checksum" in str(res[1])
    for r, j in ((res[0], good[0]), (res[2], good[1])):
        assert r.file_bytes() == [x[0] for x in oracle.compact(j, "oracle")]
