"""The allocation-free CRC entry point (lc_crc32c_noalloc), through the C ABI.

Some hosts cannot allocate device memory at the moment they need a checksum:
their device memory is owned by another allocator, or the path must not take
the implicit device synchronisation that cudaMalloc/cudaFree bring.  This
entry point takes only device pointers and keeps its scratch in a fixed
static device array.  Two calls in a row must give the same masked CRC as the
pooled entry point, lc_crc32c, on the same bytes (bit-exact: CRCs are
integers).  The file sorts last so that a failure here leaves the rest of the
suite already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LC_ERR_UNSUPPORTED = 7


@pytest.fixture(scope="module")
def lib():
    from luda_b200 import engine as eng_mod
    l = eng_mod.load_library()
    l.lc_crc32c_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    l.lc_crc32c_noalloc.restype = C.c_int
    return l


def _noalloc(lib, dev_tensor, n, out_tensor):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.lc_crc32c_noalloc(dev_tensor.data_ptr() if n else None, n, out_tensor.data_ptr(),
                               C.c_void_p(stream))
    assert st == 0, st
    torch.cuda.synchronize()
    return int(out_tensor.cpu().numpy().view(np.uint32)[0])


def test_noalloc_matches_pooled_entry_point_twice(lib, engine):
    import torch
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    for n, seed in ((5 * (1 << 20) + 13, 1), (200003, 2)):
        host = np.random.default_rng(seed).integers(0, 256, n, dtype=np.uint8)
        dev = torch.from_numpy(host).cuda()
        torch.cuda.synchronize()
        got = _noalloc(lib, dev, n, out)
        assert got == engine.crc32c(device_ptr=dev.data_ptr(), n=n)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    import torch
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    src = torch.zeros(16, dtype=torch.uint8, device="cuda")
    st = lib.lc_crc32c_noalloc(src.data_ptr(), (1 << 30) + 1, out.data_ptr(), None)
    assert st == LC_ERR_UNSUPPORTED
