"""CPU-side checks of the C ABI: the library builds for sm_100a, loads on a
host without a GPU, and exports exactly what include/vexq_cuda.h declares."""
import ctypes as C
import os
import re

import numpy as np

from vexq_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "vexq_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"^\s*(?:int32_t|const char\s*\*)\s*(vexq_\w+)\s*\(", txt, flags=re.M))


def test_header_and_binding_list_agree():
    assert declared_functions() == set(abi.EXPORTS)


def test_library_loads_and_exports_every_declared_symbol():
    build.build()
    lib = abi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.vexq_abi_version() == 1


def test_selvec_from_bits_matches_bool_to_selvec():
    # BoolToSelVecInto (exec/expr.go:1545-1564): ascending physical indices of set bits
    build.build()
    lib = abi.load()
    rng = np.random.default_rng(3)
    n = 3000
    keep = rng.random(n) < 0.3
    bits = np.packbits(keep, bitorder="little")
    buf = (C.c_uint8 * len(bits)).from_buffer_copy(bits.tobytes())
    sel = (C.c_uint16 * 1024)()
    ln = C.c_int32()
    for block in range(3):
        assert lib.vexq_selvec_from_bits(buf, n, block, sel, C.byref(ln)) == 0
        want = [i - block * 1024 for i in range(block * 1024, min(n, block * 1024 + 1024)) if keep[i]]
        assert list(sel[:ln.value]) == want


def test_errors_are_status_codes_not_crashes():
    build.build()
    lib = abi.load()
    assert lib.vexq_table_upload(None, 1, 10, 0, None) == abi.EINVAL
    assert b"null" in lib.vexq_last_error()
    assert lib.vexq_plan_run(None, 0, -1, None) == abi.EINVAL
