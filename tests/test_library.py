"""The engine's C ABI library loads and exports every entry point that
include/luda_b200.h declares (no device work: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from luda_b200 import build as lbuild
from luda_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "luda_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lc_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(engine.LIB_PATH):
        lbuild.build()
    return ctypes.CDLL(engine.LIB_PATH)


def test_header_declares_abi():
    syms = declared_symbols()
    assert set(engine.EXPORTS) <= set(syms)
    assert len(syms) >= 10


def test_library_exports_every_declared_symbol(lib):
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_version_and_status_strings(lib):
    lib.lc_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.lc_version()
    lib.lc_status_string.restype = ctypes.c_char_p
    assert lib.lc_status_string(2) == b"corruption"


def test_library_built_for_sm100a():
    # the build passes exactly one gencode: compute_100a -> sm_100a
    assert lbuild.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
