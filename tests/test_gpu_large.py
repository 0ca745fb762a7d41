"""The 1 GiB L2->L3 compactions at size on the GPU (1 + 15 tables of 64 MiB).

Run A has 8-byte keys with 1 KiB values (about 1M entries), run B 24-byte keys
with 32-byte values (about 16M entries).  Inputs are rebuilt from the seeded
generators and checked against the fixture's hashes; every output file must
have the SHA-256, size and smallest/largest keys that the reference's CPU
DoCompactionWork produced, both from host buffers and with inputs and outputs
in device memory.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

import oracle

sys.path.insert(0, os.path.dirname(__file__))
from test_oracle import golden_job, _golden  # noqa: E402

pytestmark = pytest.mark.gpu

LARGE = [c for c in _golden() if c.get("large")]


def sha(b):
    return hashlib.sha256(b).hexdigest()


@pytest.mark.parametrize("case", LARGE, ids=[c["name"] for c in LARGE])
def test_large_compaction_matches_reference(engine, oracle_lib, case):
    import torch
    job = golden_job(case)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    tables = job.input_tables()
    assert [sha(f.data) for f in tables] == case["inputs"]
    assert job.input_bytes() == case["input_bytes"]

    def check(files_bytes, res):
        assert len(files_bytes) == len(case["outputs"])
        for b, f, g in zip(files_bytes, res.files, case["outputs"]):
            assert len(b) == g["size"] and sha(b) == g["sha256"]
            assert f.smallest.hex() == g["smallest"] and f.largest.hex() == g["largest"]

    res = engine.compact(job)
    check(res.file_bytes(), res)
    assert res.bytes_in == case["input_bytes"]
    res.release()

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
    out = np.empty(dev.bytes_out, np.uint8)
    from cuda.bindings import runtime as rt
    err, = rt.cudaMemcpy(out.ctypes.data, dev.device_ptr, dev.bytes_out,
                         rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    blobs = [out[o:o + g["size"]].tobytes() for o, g in zip(dev.file_offsets, case["outputs"])]
    check(blobs, dev)
    dev.release()
    del buf
