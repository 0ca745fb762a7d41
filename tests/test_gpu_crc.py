"""lc_crc32c: masked CRC32C of a buffer on the GPU equals the reference's
crc32c::Mask(crc32c::Value(...)) (util/crc32c.h:20-32), restated in oracle/,
for host and device inputs across chunk boundaries."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 31, 32, 4095, 65535, 65536, 65537, 1 << 20, (3 << 20) + 7, 20 << 20]


def want(b: bytes) -> int:
    return oracle.crc32c_mask(oracle.crc32c(b))


def test_rfc3720_vectors(engine):
    for b in (bytes(32), b"\xff" * 32, bytes(range(32)), bytes(range(31, -1, -1))):
        assert engine.crc32c(b) == want(b)


@pytest.mark.parametrize("n", SIZES)
def test_host_buffers(engine, n):
    b = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    assert engine.crc32c(b) == want(b)


@pytest.mark.parametrize("n", SIZES)
def test_device_buffers(engine, n):
    import torch
    b = np.random.default_rng(n + 1).integers(0, 256, n, dtype=np.uint8)
    d = torch.from_numpy(b).cuda() if n else torch.zeros(1, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    assert engine.crc32c(device_ptr=d.data_ptr(), n=n) == want(b.tobytes())


def test_block_trailers_of_an_output_table(engine):
    # every block trailer the engine wrote checks out with lc_crc32c
    from luda_b200 import workloads
    job = workloads.plain_l0_l1(seed=2, scale=0.02)
    job.materialize(lambda e, o: oracle.build_table(e, o, "oracle"))
    res = engine.compact(job)
    data = bytes(res.files[0].data)
    # the index block handle from the footer, then the first data block handle
    foot = data[-48:]

    def varint(b, p):
        r, s = 0, 0
        while True:
            c = b[p]
            r |= (c & 127) << s
            p += 1
            if c < 128:
                return r, p
            s += 7
    _, p = varint(foot, 0)
    _, p = varint(foot, p)
    ioff, p = varint(foot, p)
    isize, p = varint(foot, p)
    block = data[ioff:ioff + isize + 1]
    stored = int.from_bytes(data[ioff + isize + 1:ioff + isize + 5], "little")
    assert engine.crc32c(block) == stored
