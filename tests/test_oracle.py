"""The CPU restatement (oracle/) pinned against the reference.

* Known-answer vectors from the reference's own tests:
  util/crc32c_test.cc:13-56 (RFC 3720 B.4), util/hash_test.cc:12-40,
  db/dbformat_test.cc:68-111 (separators / successors), util/bloom_test.cc
  (false-positive bound).
* Byte identity with the reference's CPU compaction through the committed
  fixtures (tests/golden/golden.json, made by the reference build) and, where
  the reference build is present, live against it.
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.job import internal_key

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.json")


@pytest.fixture(scope="module", autouse=True)
def _built(oracle_lib):
    return oracle_lib


def test_crc32c_rfc3720():
    assert oracle.crc32c(bytes(32)) == 0x8A9136AA
    assert oracle.crc32c(b"\xff" * 32) == 0x62A8AB43
    assert oracle.crc32c(bytes(range(32))) == 0x46DD794E
    assert oracle.crc32c(bytes(range(31, -1, -1))) == 0x113FDB5C
    data = bytes([0x01, 0xc0, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00,
                  0x00, 0x00, 0x00, 0x00, 0x14, 0x00, 0x00, 0x00, 0x00, 0x00, 0x04, 0x00,
                  0x00, 0x00, 0x00, 0x14, 0x00, 0x00, 0x00, 0x18, 0x28, 0x00, 0x00, 0x00,
                  0x00, 0x00, 0x00, 0x00, 0x02, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00])
    assert oracle.crc32c(data) == 0xD9963A56


def test_crc32c_mask_roundtrip():
    crc = oracle.crc32c(b"foo")
    m = oracle.crc32c_mask(crc)
    assert m != crc
    rot = (m - 0xA282EAD8) & 0xFFFFFFFF
    assert ((rot >> 17) | (rot << 15)) & 0xFFFFFFFF == crc


def test_hash_vectors():
    h = oracle.leveldb_hash
    assert h(b"", 0xBC9F1D34) == 0xBC9F1D34
    assert h(b"\x62", 0xBC9F1D34) == 0xEF1345C4
    assert h(b"\xc3\x97", 0xBC9F1D34) == 0x5B663814
    assert h(b"\xe2\x99\xa5", 0xBC9F1D34) == 0x323C078F
    assert h(b"\xe1\x80\xb9\x32", 0xBC9F1D34) == 0xED21633A
    data5 = bytes([0x01, 0xc0] + [0] * 14 + [0x14, 0, 0, 0, 0, 0, 0x04, 0, 0, 0, 0, 0x14, 0, 0,
                                              0, 0x18, 0x28, 0, 0, 0, 0, 0, 0, 0, 0x02] + [0] * 7)
    assert len(data5) == 48
    assert h(data5, 0x12345678) == 0xF333DABB


def _ik(u, s, t=1):
    return internal_key(u, s, t)


MAXSEQ = (1 << 56) - 1


def test_separator_vectors():
    sep = oracle.separator
    assert sep(_ik(b"foo", 100), _ik(b"foo", 99)) == _ik(b"foo", 100)
    assert sep(_ik(b"foo", 100), _ik(b"foo", 101)) == _ik(b"foo", 100)
    assert sep(_ik(b"foo", 100), _ik(b"foo", 100)) == _ik(b"foo", 100)
    assert sep(_ik(b"foo", 100), _ik(b"foo", 100, 0)) == _ik(b"foo", 100)
    assert sep(_ik(b"foo", 100), _ik(b"bar", 99)) == _ik(b"foo", 100)
    assert sep(_ik(b"foo", 100), _ik(b"hello", 200)) == _ik(b"g", MAXSEQ, 1)
    assert sep(_ik(b"foo", 100), _ik(b"foobar", 200)) == _ik(b"foo", 100)
    assert sep(_ik(b"foobar", 100), _ik(b"foo", 200)) == _ik(b"foobar", 100)


def test_successor_vectors():
    assert oracle.successor(_ik(b"foo", 100)) == _ik(b"g", MAXSEQ, 1)
    assert oracle.successor(_ik(b"\xff\xff", 100)) == _ik(b"\xff\xff", 100)


def test_bloom_false_positive_bound():
    # util/bloom_test.cc:110-150: FP rate <= 2% at 10 bits/key
    keys = [struct.pack("<I", i) for i in range(10000)]
    f = oracle.bloom(keys, 10)
    k = f[-1]
    bits = (len(f) - 1) * 8
    assert k == 6

    def may_match(key):
        h = oracle.leveldb_hash(key, 0xBC9F1D34)
        delta = ((h >> 17) | (h << 15)) & 0xFFFFFFFF
        for _ in range(k):
            bp = h % bits
            if not (f[bp // 8] >> (bp % 8)) & 1:
                return False
            h = (h + delta) & 0xFFFFFFFF
        return True

    assert all(may_match(x) for x in keys[:500])
    fp = sum(may_match(struct.pack("<I", i + 1000000000)) for i in range(10000))
    assert fp / 10000 <= 0.02


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def golden_job(case):
    """Rebuilds a fixture's job from its recorded generator and arguments."""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    import edge_jobs
    spec = case["spec"]
    if "edge" in spec:
        return {j.name: j for j in edge_jobs.all_cases()}[spec["edge"]]
    return getattr(workloads, spec["workload"])(**spec["kwargs"])


def sha(b):
    return hashlib.sha256(b).hexdigest()


CPU_CASES = [c for c in _golden() if c["input_bytes"] < 30 << 20]


@pytest.mark.parametrize("case", CPU_CASES, ids=[c["name"] for c in CPU_CASES])
def test_oracle_matches_reference_fixture(case):
    job = golden_job(case)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    assert [sha(f.data) for f in job.input_tables()] == case["inputs"]
    outs = oracle.compact(job, "oracle")
    assert len(outs) == len(case["outputs"])
    for (d, s, l), g in zip(outs, case["outputs"]):
        assert len(d) == g["size"]
        assert sha(d) == g["sha256"]
        assert s.hex() == g["smallest"] and l.hex() == g["largest"]


@pytest.mark.skipif(not oracle.has_ref(), reason="reference build absent")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_live(seed):
    rng = np.random.default_rng(seed)
    from luda_b200.job import TableOptions
    opts = TableOptions(block_size=int(rng.choice([1024, 2048, 4096, 16384])),
                        restart_interval=int(rng.choice([1, 3, 16, 40])),
                        bits_per_key=int(rng.choice([0, 5, 10])),
                        max_file_size=1 << 20)
    job = workloads.l0_l1_job(100 + seed, n0=int(rng.integers(1, 4)), n1=int(rng.integers(0, 3)),
                              entries_per_table=int(rng.integers(50, 6000)),
                              key_space=int(rng.choice([5000, 1 << 20])),
                              tomb_frac=float(rng.choice([0.0, 0.02, 0.3])),
                              value_len=int(rng.choice([0, 7, 100, 900])), options=opts)
    job.materialize(lambda e, o: oracle.build_table(e, o, "ref"))
    a = oracle.compact(job, "oracle")
    b = oracle.compact(job, "ref")
    assert [x[0] for x in a] == [x[0] for x in b]
    assert [(x[1], x[2]) for x in a] == [(x[1], x[2]) for x in b]


@pytest.mark.skipif(not oracle.has_ref(), reason="reference build absent")
def test_oracle_tables_readable_by_reference():
    job = workloads.plain_l0_l1(seed=9, scale=0.05)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    for (d, s, l) in oracle.compact(job, "oracle"):
        ents = oracle.read_table(d, "ref")
        assert ents[0][0] == s and ents[-1][0] == l
        assert ents == oracle.read_table(d, "oracle")


@pytest.mark.skipif(not oracle.has_ref(), reason="reference build absent")
def test_oracle_matches_reference_on_encoder_path_cases():
    # the cases tests/test_gpu_encode_paths.py runs on the GPU against the
    # restatement: here the restatement against the reference's own build
    import test_gpu_encode_paths as paths
    from luda_b200.job import TableOptions
    for ri, bs, vlen, what in paths.CASES:
        opts = TableOptions(block_size=bs, restart_interval=ri, bits_per_key=10,
                            max_file_size=1 << 20)
        job = workloads.l0_l1_job(900 + ri + vlen, n0=2, n1=2, entries_per_table=4000,
                                  key_space=1 << 20, tomb_frac=0.02, value_len=vlen,
                                  options=opts)
        job.materialize(lambda e, o: oracle.build_table(e, o, "ref"))
        inputs = [bytes(f.data) for f in job.files]
        for f in job.files:
            assert oracle.build_table(f.entries, opts, "oracle") == bytes(f.data), what
        a = oracle.compact(job, "oracle")
        b = oracle.compact(job, "ref")
        assert [x[0] for x in a] == [x[0] for x in b], what
        assert [(x[1], x[2]) for x in a] == [(x[1], x[2]) for x in b], what
        assert inputs == [bytes(f.data) for f in job.files]
