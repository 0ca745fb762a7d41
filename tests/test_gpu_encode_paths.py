"""Data-block encoder paths, compared with the CPU restatement.

The block encoder stages short pieces (up to 16 bytes, or up to 32), lists
key deltas and values of at least 33 bytes for chunk reads (at most 64 per
block, the rest staged by the lane), finds restart entries with a shift when
the restart interval is a power of two and with a division otherwise, and
writes blocks too large for its stage directly.  Each case below drives one
of those paths through a whole compaction and through the flush encoder; the
output must equal the restatement's byte for byte (which is pinned to the
reference's CPU compaction, tests/test_oracle.py).
"""
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.job import TableOptions

pytestmark = pytest.mark.gpu

# (restart interval, block size, value length, what it drives)
CASES = [
    (3, 4096, 34, "division path; about 90 values of 34 bytes per block: the long-stretch list overflows"),
    (5, 2048, 16, "division path; 16-byte values and key deltas staged in the 16-byte form"),
    (40, 4096, 17, "division path; 17-byte values staged in the 32-byte form"),
    (16, 16384, 33, "values at the long-stretch threshold, listed"),
    (7, 1024, 900, "division path; long values cut at both edges, blocks of one or two entries"),
    (16, 4096, 0, "empty values"),
    (12, 65536, 100, "blocks larger than the stage: the direct path"),
]


@pytest.mark.parametrize("ri,bs,vlen,what", CASES, ids=[f"r{c[0]}_b{c[1]}_v{c[2]}" for c in CASES])
def test_encoder_paths_match_restatement(engine, oracle_lib, ri, bs, vlen, what):
    opts = TableOptions(block_size=bs, restart_interval=ri, bits_per_key=10,
                        max_file_size=1 << 20)
    job = workloads.l0_l1_job(900 + ri + vlen, n0=2, n1=2, entries_per_table=4000,
                              key_space=1 << 20, tomb_frac=0.02, value_len=vlen, options=opts)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    for f in job.files:
        assert engine.build_table(f.entries, opts) == f.data, what
    res = engine.compact(job)
    want = oracle.compact(job, "oracle")
    assert res.file_bytes() == [w[0] for w in want], what
    assert [(f.smallest, f.largest) for f in res.files] == [(w[1], w[2]) for w in want]
