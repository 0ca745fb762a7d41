"""The block encoder's row-interleaved CRC32C, restated on the CPU.

The data-block encoder (k_encode_blocks) computes each block's trailer CRC
over a grid of 16-byte chunks that starts at the 16-byte boundary at or below
the block: lane l of a warp takes chunks l, l + 32, ... and keeps a register
u <- H(x ^ u), where H(x) is the raw CRC register after the 16 bytes x and
the row's other 496 bytes as zeros, from 0 (H is the xor of one table entry
per 5-bit field of x).  The grid bytes outside the message (block plus type
byte) are zero, every lane's register is moved back to the message's end
(x^(-8n) for the n bytes it was carried past it), the lanes' registers are
xored, and the initial all-ones register enters last as its own register
carried over the message's length.

This test rebuilds those tables the way the engine does and runs that
arithmetic in Python for messages at every 16-byte phase, against the plain
CRC32C of the restatement (oracle/lsm_oracle.c, pinned to RFC 3720 vectors in
test_oracle.py).  It checks the arithmetic only; the kernel itself is checked
byte for byte on the GPU.
"""
import numpy as np
import pytest

import oracle

POLY = 0x82F63B78
FIELD_BITS, FIELDS, ROW = 5, 26, 512


def _byte_step(c, b):
    c ^= b
    for _ in range(8):
        c = (c >> 1) ^ POLY if c & 1 else c >> 1
    return c


def _raw(c, data):
    for b in data:
        c = _byte_step(c, b)
    return c


def _mulmod(a, b):
    # reflected GF(2) product mod P: bit 31 is x^0
    p = 0
    for _ in range(32):
        if a & 0x80000000:
            p ^= b
        a = (a << 1) & 0xFFFFFFFF
        b = (b >> 1) ^ POLY if b & 1 else b >> 1
    return p


def _build_tables():
    zeros = bytes(ROW - 16)
    h5 = np.zeros((FIELDS, 1 << FIELD_BITS), np.uint32)
    for i in range(FIELDS):
        for v in range(1 << FIELD_BITS):
            x = 0
            for bit in range(FIELD_BITS):
                at = FIELD_BITS * i + bit
                if (v >> bit) & 1 and at < 128:
                    x |= 1 << at
            h5[i, v] = _raw(_raw(0, x.to_bytes(16, "little")), zeros)
    # x^(-8n): the shift that undoes n zero bytes, by inverting one zero-byte step
    by_top = {}
    for i in range(256):
        by_top[_byte_step(0, i) >> 24] = i
    xinv, c = [], 0x80000000
    for _ in range(ROW):
        xinv.append(c)
        i = by_top[c >> 24]
        c = (((c ^ _byte_step(0, i)) << 8) & 0xFFFFFFFF) | i
    ones, c = [], 0xFFFFFFFF
    for _ in range(8192):
        ones.append(c)
        c = _byte_step(c, 0)
    return h5, xinv, ones


@pytest.fixture(scope="module")
def tables():
    return _build_tables()


def _h(h5, x16):
    v = int.from_bytes(x16, "little")
    r = 0
    for i in range(FIELDS):
        r ^= int(h5[i, (v >> (FIELD_BITS * i)) & ((1 << FIELD_BITS) - 1)])
    return r


def _rows_crc(tables, block: bytes, phase: int) -> int:
    h5, xinv, ones = tables
    msg = block + b"\x00"  # the type byte of an uncompressed block
    m0, m1 = phase, phase + len(msg)
    grid = bytearray((m1 + 15) // 16 * 16)
    grid[m0:m1] = msg
    v = 0
    for lane in range(32):
        u, last = 0, None
        for p in range(16 * lane, m1, ROW):
            x = bytearray(grid[p:p + 16])
            x[0:4] = (int.from_bytes(x[0:4], "little") ^ u).to_bytes(4, "little")
            u = _h(h5, bytes(x))
            last = p
        if last is not None:
            v ^= _mulmod(u, xinv[last + ROW - m1])
    full = v ^ ones[m1 - m0] ^ 0xFFFFFFFF
    return (((full >> 15) | (full << 17)) + 0xA282EAD8) & 0xFFFFFFFF


def test_row_crc_matches_crc32c(oracle_lib, tables):
    rng = np.random.default_rng(11)
    for n in (4, 11, 15, 16, 17, 100, 511, 512, 513, 1500, 4200):
        block = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        want = oracle.crc32c_mask(oracle.crc32c(block + b"\x00"))
        for phase in range(16):
            assert _rows_crc(tables, block, phase) == want, (n, phase)


def test_row_crc_needs_the_initial_register(oracle_lib, tables):
    # without the all-ones register's share the trailer is wrong: the term is
    # what replaces inverting the message's first four bytes
    h5, xinv, _ = tables
    block = bytes(range(200))
    want = oracle.crc32c_mask(oracle.crc32c(block + b"\x00"))
    assert _rows_crc(tables, block, 5) == want
    assert _rows_crc((h5, xinv, [0] * len(tables[2])), block, 5) != want


def _xpow8(n):
    # x^(8n) mod P by square and multiply (reflected; x^8 is one zero byte from x^0)
    r, base = 0x80000000, _byte_step(0x80000000, 0)
    while n:
        if n & 1:
            r = _mulmod(r, base)
        base = _mulmod(base, base)
        n >>= 1
    return r


def test_long_shift_is_a_product_of_two_table_entries():
    # the meta-block CRC moves each 4 KiB piece's register to its block's end
    # by x^(8n), n = 8192 hi + lo, as xpow[lo] * xpow_hi[hi]; the engine builds
    # xpow_hi[h] as xpow_hi[h - 1] * (xpow[8191] * xpow[1])
    N = 8192
    xpow = [0x80000000]
    for _ in range(N - 1):
        xpow.append(_byte_step(xpow[-1], 0))
    step = _mulmod(xpow[N - 1], xpow[1])
    assert step == _xpow8(N)
    hi_tab = [0x80000000]
    for _ in range(64):
        hi_tab.append(_mulmod(hi_tab[-1], step))
    rng = np.random.default_rng(5)
    for n in [0, 1, N - 1, N, N + 1, 40 * N + 17] + rng.integers(0, 64 * N, 20).tolist():
        hi, lo = divmod(int(n), N)
        assert _mulmod(xpow[lo], hi_tab[hi]) == _xpow8(int(n)), n
