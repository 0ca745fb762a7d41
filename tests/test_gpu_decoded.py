"""Decoded runs kept on the device between chained compactions.

A first compaction keeps its outputs on the device together with their
decoded entries (keep_decoded).  A second compaction reads those outputs as
level-1 inputs, together with new level-0 tables, from device memory: once
from their decoded form (no parse, no decode) and once encoded.  Both must
give the same bytes, equal to the CPU restatement's; a descriptor that pairs
a decoded form with a table of another size is refused.
"""
import numpy as np
import pytest

import oracle
from luda_b200 import workloads
from luda_b200.engine import LcError
from luda_b200.job import CompactionJob, Entries, FileMeta, TableOptions, internal_key

pytestmark = pytest.mark.gpu

OPTS = TableOptions(max_file_size=96 << 10)


def _new_l0(seed, seq0, n, key_space):
    rng = np.random.default_rng(seed)
    ids = np.unique(rng.integers(0, key_space, n))
    keys, vals = [], []
    for i, u in enumerate(ids.tolist()):
        vtype = 0 if rng.random() < 0.05 else 1
        keys.append(internal_key(b"%016d" % u, seq0 + i, vtype))
        vals.append(b"" if vtype == 0 else rng.integers(0, 256, 100, dtype=np.uint8).tobytes())
    return Entries.from_lists(keys, vals), seq0 + len(ids)


def _device_copy(torch, blobs):
    offs, total = [], 0
    for b in blobs:
        offs.append(total)
        total += (len(b) + 15) // 16 * 16
    buf = torch.zeros(total + 16, dtype=torch.uint8, device="cuda")
    for b, o in zip(blobs, offs):
        buf[o:o + len(b)] = torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()
    return buf, [buf.data_ptr() + o for o in offs]


@pytest.mark.parametrize("seed", [1, 2])
def test_chained_job_reads_decoded_outputs(engine, seed):
    import torch
    first = workloads.l0_l1_job(seed, n0=2, n1=2, entries_per_table=4000, key_space=1 << 16,
                                options=OPTS, name="first")
    first.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    r1 = engine.run(engine.prepare(first, outputs_on_device=2, keep_decoded=True))
    assert len(r1.files) >= 3 and all(f.decoded for f in r1.files)
    # second job: new level-0 tables over the first job's outputs (level 1)
    files, number, seq = [], 100, first.last_sequence + 1
    for k in range(2):
        e, seq = _new_l0(seed * 10 + k, seq, 3000, 1 << 16)
        files.append(FileMeta(0, number, e.key(0), e.key(e.n - 1), entries=e))
        number += 1
    for f in r1.files:
        files.append(FileMeta(1, number, f.smallest, f.largest, data=bytes(f.data),
                              file_size=len(f.data)))
        number += 1
    second = CompactionJob(level=0, files=files, snapshots=[], last_sequence=seq - 1,
                           options=OPTS, name="second")
    second.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    tables = second.input_tables()
    # level-0 tables uploaded; level-1 tables are the first job's device outputs
    l0 = [f for f in tables if f.level == 0]
    buf, l0_ptrs = _device_copy(torch, [f.data for f in l0])
    by_number = {f.number: i for i, f in enumerate(files)}
    ptrs, decoded = [], []
    for f in tables:
        if f.level == 0:
            ptrs.append(l0_ptrs[l0.index(f)])
            decoded.append(None)
        else:
            i = by_number[f.number] - 2
            ptrs.append(r1.device_ptr + r1.file_offsets[i])
            decoded.append(r1.files[i].decoded)
    torch.cuda.synchronize()
    want = [o[0] for o in oracle.compact(second, "oracle")]
    plain = engine.run(engine.prepare(second, device_tables=ptrs))
    cached = engine.run(engine.prepare(second, device_tables=ptrs, decoded=decoded))
    assert cached.decoded_inputs == len(r1.files) and plain.decoded_inputs == 0
    assert plain.file_bytes() == want
    assert cached.file_bytes() == want
    assert [(f.smallest, f.largest) for f in cached.files] == \
        [(f.smallest, f.largest) for f in plain.files]
    plain.release()
    cached.release()
    # a decoded form paired with a table of another size is refused
    wrong = list(decoded)
    j = next(i for i, d in enumerate(decoded) if d)
    k = next(i for i, d in enumerate(decoded) if d and
             len(r1.files[by_number[tables[i].number] - 2].data) !=
             len(r1.files[by_number[tables[j].number] - 2].data))
    wrong[j], wrong[k] = decoded[k], decoded[j]
    with pytest.raises(LcError):
        engine.run(engine.prepare(second, device_tables=ptrs, decoded=wrong))
    r1.release()
    del buf
