"""amx_filter_compressstore_noalloc: the fused filter + compressstore for callers that cannot
allocate device memory (for example an engine whose memory pool is fully handed out, or code on a
path where cudaMalloc is forbidden because it can synchronise the device).  It uses a fixed
scratch array inside the library instead of a caller workspace.

Checked through the C ABI against the workspace-taking entry point, bit-exact (integer data has
no tolerance), on two calls in a row so that the second call starts from the first call's
leftover scratch.  This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import SLAB, NOGAPS, PLAIN32, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu


def _noalloc_entry():
    from amethyst_b200 import _capi as A
    from amethyst_b200 import build

    h = C.CDLL(build.LIB)
    f = h.amx_filter_compressstore_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(A.Column), C.POINTER(A.Predicate), C.POINTER(A.Column), C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("fmt,bits,n,kind,k0", [
    (SLAB, 11, (1 << 20) + 77, 1, 205),    # v < 205 on 11-bit slabs
    (SLAB, 3, 300001, 4, 5),               # v >= 5 on 3-bit slabs
    (NOGAPS, 21, 123457, 7, 1000),         # 1000 <= v <= k1 on a gap-free stream
    (PLAIN32, 32, 99999, 6, 12345),        # v != 12345 on plain words
])
def test_noalloc_matches_workspace_entry_point(cuda, fmt, bits, n, kind, k0):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    f = _noalloc_entry()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    k1 = (1 << 20) if kind == 7 else 0
    p = ops.predicate(kind, k0, k1, bits)
    for call in range(2):
        v, raw = make_column(1000 * call + bits + n, fmt, bits, n)
        col = to_gpu(raw, n, fmt, bits)
        want_out, want_cnt = ops.filter_compressstore(col, p, fmt, bits)
        out = ops.PackedColumn.empty(n, fmt, bits)
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        st = f(C.byref(col.desc), C.byref(p), C.byref(out.desc), C.c_void_p(cnt.data_ptr()), stream)
        assert st == 0, A.lib().amx_last_error()
        torch.cuda.synchronize()
        c = int(cnt[0].item())
        assert c == int(want_cnt[0].item())
        assert np.array_equal(gpu_bytes(out, c), gpu_bytes(want_out, c))


def test_noalloc_rejects_columns_over_the_scratch_limit(cuda):
    from amethyst_b200 import _capi as A

    f = _noalloc_entry()
    big = A.Column(C.c_void_p(0x10000), (1 << 29) + 1, A.SLAB, 11)
    out = A.Column(C.c_void_p(0x20000), (1 << 29) + 1, A.SLAB, 11)
    p = A.Predicate(A.PRED_LT, 11, 205, 0)
    assert f(C.byref(big), C.byref(p), C.byref(out), C.c_void_p(0x30000), None) == 7
    assert b"2^29" in A.lib().amx_last_error()


def test_noalloc_status_reports_a_device_side_timeout(cuda):
    """A bounded look-back wait made to run out (amx_test_lookback_timeout) on the no-alloc path
    is reported by amx_filter_compressstore_noalloc_status; the next call clears the record and
    is bit-exact again."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import build, ops

    h = C.CDLL(build.LIB)
    status = h.amx_filter_compressstore_noalloc_status
    status.restype = C.c_int
    status.argtypes = [C.c_void_p]
    f = _noalloc_entry()
    L = A.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 1 << 21
    v, raw = make_column(4242, SLAB, 11, n)
    col = to_gpu(raw, n, SLAB, 11)
    p = ops.predicate(A.PRED_LT, 205, 0, 11)
    want_out, want_cnt = ops.filter_compressstore(col, p, SLAB, 11)
    out = ops.PackedColumn.empty(n, SLAB, 11)
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    try:
        A.check(L.amx_test_lookback_timeout(0, 2000))
        assert f(C.byref(col.desc), C.byref(p), C.byref(out.desc), C.c_void_p(cnt.data_ptr()), stream) == 0
        assert status(stream) == 6
    finally:
        L.amx_test_lookback_timeout((1 << 64) - 1, 0)
    assert f(C.byref(col.desc), C.byref(p), C.byref(out.desc), C.c_void_p(cnt.data_ptr()), stream) == 0
    assert status(stream) == 0
    c = int(cnt[0].item())
    assert c == int(want_cnt[0].item())
    assert np.array_equal(gpu_bytes(out, c), gpu_bytes(want_out, c))
