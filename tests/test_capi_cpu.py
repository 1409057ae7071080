"""C ABI checks that need no GPU: the library loads, exports every entry point declared in
include/*.h, and rejects bad arguments with status codes before touching the device."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from amethyst_b200 import build

    if not os.path.exists(build.LIB):
        build.build()
    from amethyst_b200 import _capi

    return _capi.lib()


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(amx_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(lib):
    from amethyst_b200 import build

    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    decl = declared_functions()
    assert len(decl) >= 15
    missing = [d for d in decl if d not in exported]
    assert not missing, missing


def test_sizing_helpers(lib):
    from amethyst_b200 import _capi as A

    assert lib.amx_version() >= 100
    assert lib.amx_storage_bytes(A.SLAB, 11, 10) == 16
    assert lib.amx_storage_bytes(A.SLAB, 11, 2**24) == 26843552
    assert lib.amx_storage_bytes(A.NOGAPS, 11, 64) == 88
    assert lib.amx_storage_bytes(A.PLAIN32, 11, 3) == 12
    assert lib.amx_storage_bytes(A.PLAIN32, 33, 3) == 0  # invalid width
    assert lib.amx_mask_bytes(33) == 8
    assert lib.amx_binary_out_bits(A.OP_ADD, 7, 13) == 14
    assert lib.amx_binary_out_bits(A.OP_MUL, 40, 40) == 64
    assert lib.amx_workspace_bytes(1 << 20) >= 64 + 8 * 256


def test_argument_errors(lib):
    from amethyst_b200 import _capi as A

    ws = (C.c_uint8 * 4096)()
    good = A.Column(C.c_void_p(0x10000), 100, A.SLAB, 11)
    bad_fmt = A.Column(C.c_void_p(0x10000), 100, 9, 11)
    bad_w = A.Column(C.c_void_p(0x10000), 100, A.PLAIN32, 40)
    misal = A.Column(C.c_void_p(0x10008), 100, A.SLAB, 11)
    pred = A.Predicate(A.PRED_LT, 0, 5, 0)
    assert lib.amx_filter(None, C.byref(pred), C.c_void_p(0x20000), ws, 4096, None) == 1
    assert lib.amx_filter(C.byref(bad_fmt), C.byref(pred), C.c_void_p(0x20000), ws, 4096, None) == 1
    assert lib.amx_filter(C.byref(bad_w), C.byref(pred), C.c_void_p(0x20000), ws, 4096, None) == 1
    assert lib.amx_filter(C.byref(misal), C.byref(pred), C.c_void_p(0x20000), ws, 4096, None) == 3
    assert b"aligned" in lib.amx_last_error()
    assert lib.amx_filter(C.byref(good), None, C.c_void_p(0x20000), ws, 4096, None) == 1
    bad_pred = A.Predicate(77, 0, 0, 0)
    assert lib.amx_filter(C.byref(good), C.byref(bad_pred), C.c_void_p(0x20000), ws, 4096, None) == 1
    small_out = A.Column(C.c_void_p(0x30000), 50, A.SLAB, 11)
    assert lib.amx_filter_compressstore(C.byref(good), C.byref(pred), C.byref(small_out), None, ws, 4096, None) == 1
    other = A.Column(C.c_void_p(0x40000), 99, A.SLAB, 11)
    out = A.Column(C.c_void_p(0x30000), 100, A.SLAB, 12)
    assert lib.amx_binary(A.OP_ADD, C.byref(good), C.byref(other), C.byref(out), ws, 4096, None) == 1
    assert lib.amx_binary(99, C.byref(good), C.byref(good), C.byref(out), ws, 4096, None) == 1
    assert lib.amx_reduce(9, C.byref(good), None, C.c_void_p(0x50000), ws, 4096, None) == 1
    huge = A.Column(C.c_void_p(0x10000), 1 << 41, A.SLAB, 11)
    assert lib.amx_reduce(0, C.byref(huge), None, C.c_void_p(0x50000), ws, 4096, None) == 7
    # workspace too small is caught before any launch
    assert lib.amx_reduce(0, C.byref(good), None, C.c_void_p(0x50000), ws, 8, None) == 4
    assert lib.amx_reduce(0, C.byref(good), None, C.c_void_p(0x50000), None, 0, None) == 4


def test_status_strings(lib):
    for s in range(8):
        assert lib.amx_status_string(s)
