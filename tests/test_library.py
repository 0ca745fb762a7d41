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


def test_ctypes_structs_match_header_layout():
    """Every ctypes mirror of a header struct has the C size and field offsets
    (a small C program compiled against the header prints them)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = [("lc_config", engine.LcConfig), ("lc_engine_stats", engine.LcEngineStats),
             ("lc_tuning", engine.LcTuning), ("lc_table", engine.LcTable),
             ("lc_file_range", engine.LcFileRange), ("lc_table_options", engine.LcTableOptions),
             ("lc_job_desc", engine.LcJobDesc), ("lc_job_out", engine.LcJobOut)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "luda_b200.h"',
             "int main(void) {"]
    want = []
    for cname, py in pairs:
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(py))
        for f in py._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {f[0]}));')
            want.append(getattr(py, f[0]).offset)
    lines += ["  return 0;", "}"]
    out_dir = os.path.join(ROOT, "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "abi_layout")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), "-x", "c", "-",
                    "-o", exe], input="\n".join(lines).encode(), check=True)
    got = [int(x) for x in subprocess.run([exe], capture_output=True, check=True).stdout.split()]
    assert got == want


def test_two_gib_job_is_admitted_under_default_budget(lib):
    """lc_estimate_device_bytes only reads the descriptor (no device work): a
    job of 32 tables of 64 MiB (2 GiB) from host memory is admitted under the
    default 40 GiB budget, and the estimate grows with the input."""
    lib.lc_estimate_device_bytes.argtypes = [ctypes.POINTER(engine.LcJobDesc),
                                             ctypes.POINTER(ctypes.c_uint64)]
    lib.lc_estimate_device_bytes.restype = ctypes.c_int
    dummy = ctypes.create_string_buffer(16)  # never read: only the sizes count

    def estimate(n_tables, table_bytes):
        tabs = (engine.LcTable * n_tables)()
        for t in tabs:
            t.data = ctypes.addressof(dummy)
            t.size = table_bytes
        runs = (ctypes.c_int32 * 2)(1, n_tables - 1)
        d = engine.LcJobDesc()
        d.level, d.n_tables, d.tables, d.n_runs, d.run_table_count = 1, n_tables, tabs, 2, runs
        d.options = engine.LcTableOptions(4096, 16, 10, 64 << 20)
        v = ctypes.c_uint64()
        assert lib.lc_estimate_device_bytes(ctypes.byref(d), ctypes.byref(v)) == 0
        return v.value

    two_gib = estimate(32, 64 << 20)
    assert 2 << 30 < two_gib < 40 << 30
    assert estimate(16, 64 << 20) < two_gib
