"""C ABI checks of the matrix multiply, group-by, batch and selector entry points that need no GPU:
sizing functions, and argument errors that every entry point reports with a status code before
it touches the device (the pointers below are never dereferenced)."""
import ctypes as C

import pytest


@pytest.fixture(scope="module")
def lib():
    import os

    from amethyst_b200 import build

    if not os.path.exists(build.LIB):
        build.build()
    from amethyst_b200 import _capi

    return _capi.lib()


def col(ptr, n, fmt, bits):
    from amethyst_b200 import _capi as A

    return A.Column(C.c_void_p(ptr), n, fmt, bits)


def test_matmul_sizing(lib):
    from amethyst_b200 import _capi as A

    # u7 x u7 at K = 4096: the widest product 4096 * 127^2 = 66,064,384 needs 26 bits (2 per slab)
    assert lib.amx_matmul_out_bytes(A.SLAB, 0, 4096, 4096, 4096, 7, 7) == 8 * 4096 * 2048
    assert lib.amx_matmul_out_bytes(A.PLAIN32, 0, 3, 5, 7, 8, 8) == 4 * 15
    assert lib.amx_matmul_out_bytes(A.NOGAPS, 20, 2, 3, 9, 8, 8) == 8 * ((6 * 20 + 63) // 64)
    assert lib.amx_matmul_out_bytes(A.SLAB, 0, 4, 4, 4, 9, 8) == 0  # entries wider than 8 bits
    assert lib.amx_matmul_out_bytes(A.PLAIN32, 40, 4, 4, 4, 8, 8) == 0  # plain32 holds 32 bits
    ws = lib.amx_matmul_workspace_bytes(4096, 4096, 4096)
    # header + A (4096 x 4096 u8) + B^T (4096 x 4096 u8) + C (4096 x 4096 int32)
    assert ws >= 1024 + 2 * 4096 * 4096 + 4 * 4096 * 4096 and ws % 1024 == 0


def test_matmul_argument_errors(lib):
    from amethyst_b200 import _capi as A

    a = col(0x100000, 4 * 8, A.SLAB, 7)
    b = col(0x200000, 8 * 5, A.SLAB, 7)
    out = col(0x300000, 4 * 5, A.PLAIN32, 32)
    ws = C.c_void_p(0x400000)
    nb = lib.amx_matmul_workspace_bytes(4, 5, 8)
    call = lambda a_, b_, m, n, k, o, w=ws, wb=nb: lib.amx_matmul(C.byref(a_), C.byref(b_), m, n, k,  # noqa: E731
                                                                    C.byref(o) if o is not None else None, None,
                                                                    w, wb, None)
    assert call(a, b, 4, 5, 8, None) == 1                           # no output column
    assert call(a, b, 4, 5, 7, out) == 1                            # a holds 32 entries, M*K = 28
    assert call(a, b, 4, 5, 8, col(0x300000, 19, A.PLAIN32, 32)) == 1  # output capacity below M*N
    assert call(col(0x100000, 32, A.SLAB, 9), b, 4, 5, 8, out) == 2  # 9-bit entries
    assert call(a, b, 4, 5, 8, col(0x300008, 20, A.PLAIN32, 32)) == 3  # misaligned output
    assert call(a, b, 4, 5, 8, out, None, 0) == 4                   # no workspace
    assert call(a, b, 4, 5, 8, out, ws, nb - 1) == 4                # workspace too small
    assert call(a, b, 4, 5, 8, out, C.c_void_p(0x400100), nb) == 3  # workspace not 1024-aligned
    big_a = col(0x100000, 40000, A.PLAIN32, 8)
    big_b = col(0x200000, 40000, A.PLAIN32, 8)
    assert lib.amx_matmul(C.byref(big_a), C.byref(big_b), 1, 1, 40000, C.byref(out), None, ws,
                          lib.amx_matmul_workspace_bytes(1, 1, 40000), None) == 2  # int32 could overflow


def test_groupby_sizing_and_errors(lib):
    from amethyst_b200 import _capi as A

    assert lib.amx_groupby_workspace_bytes(0) == 0
    assert lib.amx_groupby_workspace_bytes(25) == 0
    w10 = lib.amx_groupby_workspace_bytes(10)
    assert w10 >= 2 * 8 * 1024 and w10 % 256 == 0
    keys = col(0x100000, 100, A.SLAB, 10)
    vals = col(0x200000, 100, A.SLAB, 16)
    out = col(0x300000, 1024, A.PLAIN64, 64)
    g = C.c_void_p(0x500000)
    call = lambda k, v, w, wb: lib.amx_groupby(C.byref(k), C.byref(v), None, C.byref(out), C.byref(out),  # noqa: E731
                                               C.byref(out), g, w, wb, None)
    assert call(col(0x100000, 100, A.SLAB, 33), vals, C.c_void_p(0x400000), 1 << 30) == 2  # keys over 32 bits
    wide = col(0x100000, 100, A.SLAB, 25)
    assert call(wide, vals, C.c_void_p(0x400000), 4096) == 4                             # no hash table fits
    assert call(wide, vals, C.c_void_p(0x400010), 1 << 30) == 3                          # not 256-byte aligned
    w25 = lib.amx_groupby_wide_workspace_bytes(25, 1000)
    assert w25 > 8 * 2048 * 3 + (1 << 25) // 8 and w25 % 256 == 0                        # 2048 slots, 4 MB bitmap
    assert lib.amx_groupby_wide_workspace_bytes(24, 1000) == 0                           # dense keys: the other call
    assert lib.amx_groupby_wide_workspace_bytes(33, 1000) == 0
    assert call(keys, col(0x200000, 99, A.SLAB, 16), C.c_void_p(0x400000), w10) == 1    # lengths differ
    assert call(keys, vals, C.c_void_p(0x400000), w10 - 1) == 4                          # workspace too small
    assert call(keys, vals, C.c_void_p(0x400010), w10) == 3                              # not 256-byte aligned
    small = col(0x300000, 1000, A.PLAIN64, 64)
    assert lib.amx_groupby(C.byref(keys), C.byref(vals), None, C.byref(small), None, None, g,
                           C.c_void_p(0x400000), w10, None) == 1                          # capacity below 2^10


def test_batch_sizing_and_errors(lib):
    from amethyst_b200 import _capi as A

    ins = (A.Column * 2)(col(0x100000, 1000, A.SLAB, 11), col(0x200000, 5000, A.SLAB, 3))
    assert lib.amx_batch_workspace_bytes(ins, 2, None) > 0
    t512 = A.BatchTuning(512, 0)
    assert lib.amx_batch_workspace_bytes(ins, 2, C.byref(t512)) > 0
    mixed = (A.Column * 1)(col(0x100000, 1000, A.PLAIN32, 11))
    assert lib.amx_batch_workspace_bytes(mixed, 1, None) == 0  # slab columns only
    preds = (A.Predicate * 2)(A.Predicate(A.PRED_LT, 11, 5, 0), A.Predicate(A.PRED_LT, 3, 2, 0))
    outs = (A.Column * 2)(col(0x300000, 1000, A.SLAB, 11), col(0x400000, 5000, A.SLAB, 3))
    plan = A.BatchPlan()
    ws = C.c_void_p(0x500000)
    nb = lib.amx_batch_workspace_bytes(ins, 2, None)
    assert lib.amx_batch_prepare(ins, preds, outs, 2, None, None, ws, nb, None) == 1        # no plan
    wrong_w = (A.Column * 2)(col(0x300000, 1000, A.SLAB, 12), col(0x400000, 5000, A.SLAB, 3))
    assert lib.amx_batch_prepare(ins, preds, wrong_w, 2, None, C.byref(plan), ws, nb, None) == 2
    short = (A.Column * 2)(col(0x300000, 999, A.SLAB, 11), col(0x400000, 5000, A.SLAB, 3))
    assert lib.amx_batch_prepare(ins, preds, short, 2, None, C.byref(plan), ws, nb, None) == 1
    assert lib.amx_batch_prepare(mixed, preds, outs, 1, None, C.byref(plan), ws, nb, None) == 2
    assert lib.amx_batch_prepare(ins, preds, outs, 2, None, C.byref(plan), ws, nb - 1, None) == 4
    assert lib.amx_batch_prepare(ins, preds, outs, 2, None, C.byref(plan), C.c_void_p(0x500010), nb, None) == 3
    assert lib.amx_batch_run(None, None, None, ws, nb, None) == 1


def test_selector_network_sizing_and_errors(lib):
    assert lib.amx_mlp_param_count(4) == 16 * 64 + 64 + 64 * 64 + 64 + 4 * 64 + 4
    assert lib.amx_mlp_param_count(8) == 16 * 64 + 64 + 64 * 64 + 64 + 8 * 64 + 8
    assert lib.amx_mlp_param_count(1) == 0 and lib.amx_mlp_param_count(9) == 0
    p = C.c_void_p(0x100000)
    assert lib.amx_mlp_forward(p, 9, p, 4, p, None) == 1
    assert lib.amx_mlp_forward(None, 4, p, 4, p, None) == 1
    assert lib.amx_mlp_train_step(p, p, 0, 4, p, p, 4, C.c_float(0.01), None, None) == 1  # steps count from 1
    assert lib.amx_mlp_train_step(p, None, 1, 4, p, p, 4, C.c_float(0.01), None, None) == 1


def test_noalloc_rejects_oversized_columns_before_any_device_work(lib):
    from amethyst_b200 import _capi as A

    big = col(0x100000, (1 << 29) + 1, A.SLAB, 11)
    out = col(0x200000, (1 << 29) + 1, A.SLAB, 11)
    pred = A.Predicate(A.PRED_LT, 11, 205, 0)
    assert lib.amx_filter_compressstore_noalloc(C.byref(big), C.byref(pred), C.byref(out), None, None) == 7
    assert b"2^29" in lib.amx_last_error()


def test_groupby_sort_sizing_and_errors(lib):
    """amx_groupby_sort: workspace sizes (two copies of the pairs, one of the groups) and the
    argument checks that return before any device work."""
    from amethyst_b200 import _capi as A

    assert lib.amx_groupby_sort_workspace_bytes(1000, 0, 16) == 0
    assert lib.amx_groupby_sort_workspace_bytes(1000, 33, 16) == 0
    assert lib.amx_groupby_sort_workspace_bytes(1000, 32, 65) == 0
    w32 = lib.amx_groupby_sort_workspace_bytes(1 << 20, 32, 16)
    w64 = lib.amx_groupby_sort_workspace_bytes(1 << 20, 32, 40)
    assert w32 % 256 == 0 and w32 >= (1 << 20) * (2 * 4 + 2 * 4 + 4 + 8 + 8)
    assert w64 >= w32 + (1 << 20) * 8  # 64-bit values carried for values over 32 bits
    assert lib.amx_groupby_sort_workspace_bytes(0, 10, 10) > 0
    keys = col(0x100000, 100, A.SLAB, 10)
    vals = col(0x200000, 100, A.SLAB, 16)
    out = col(0x300000, 100, A.PLAIN64, 64)
    g = C.c_void_p(0x500000)
    w = lib.amx_groupby_sort_workspace_bytes(100, 10, 16)
    call = lambda k, v, ws, wb: lib.amx_groupby_sort(C.byref(k), C.byref(v), None, C.byref(out), C.byref(out),  # noqa: E731
                                                     C.byref(out), g, ws, wb, None)
    assert call(col(0x100000, 100, A.SLAB, 33), vals, C.c_void_p(0x400000), 1 << 30) == 2  # keys over 32 bits
    assert call(keys, col(0x200000, 99, A.SLAB, 16), C.c_void_p(0x400000), w) == 1       # lengths differ
    assert call(keys, vals, C.c_void_p(0x400000), w - 1) == 4                            # workspace too small
    assert call(keys, vals, C.c_void_p(0x400010), w) == 3                                # not 256-byte aligned
    assert lib.amx_groupby_sort_status(None, None) == 1
