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
MASK_OF_EMPTY = 0xa282ead8  # crc32c::Mask(crc32c::Value("", 0))


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


def test_noalloc_empty_buffer(lib):
    import torch
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    assert _noalloc(lib, None, 0, out) == MASK_OF_EMPTY


def test_noalloc_back_to_back_on_one_stream(lib, engine):
    """Three calls queued on one stream with no wait in between: each clears
    the shared ticket counter before its own launch."""
    import torch
    sizes = (3 * (1 << 20) + 5, 777, 9 * (1 << 20))
    bufs, outs = [], []
    for k, n in enumerate(sizes):
        host = np.random.default_rng(10 + k).integers(0, 256, n, dtype=np.uint8)
        bufs.append(torch.from_numpy(host).cuda())
        outs.append(torch.zeros(4, dtype=torch.uint8, device="cuda"))
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for b, o, n in zip(bufs, outs, sizes):
        assert lib.lc_crc32c_noalloc(b.data_ptr(), n, o.data_ptr(), C.c_void_p(stream)) == 0
    torch.cuda.synchronize()
    for b, o, n in zip(bufs, outs, sizes):
        got = int(o.cpu().numpy().view(np.uint32)[0])
        assert got == engine.crc32c(device_ptr=b.data_ptr(), n=n)


def test_noalloc_largest_accepted_size(lib, engine):
    """Exactly the 1 GiB limit (every chunk register of the static array)."""
    import torch
    n = 1 << 30
    free, _ = torch.cuda.mem_get_info()
    if free < 3 * n:
        pytest.skip("not enough free device memory for a 1 GiB buffer")
    dev = torch.empty(n, dtype=torch.uint8, device="cuda")
    dev.random_(0, 256, generator=torch.Generator("cuda").manual_seed(5))
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    got = _noalloc(lib, dev, n, out)
    assert got == engine.crc32c(device_ptr=dev.data_ptr(), n=n)
    del dev


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    import torch
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    src = torch.zeros(16, dtype=torch.uint8, device="cuda")
    st = lib.lc_crc32c_noalloc(src.data_ptr(), (1 << 30) + 1, out.data_ptr(), None)
    assert st == LC_ERR_UNSUPPORTED
    assert b"1 GiB" in lib.lc_last_error()
