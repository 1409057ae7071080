"""The packed-integer matrix multiply (integer tensor cores) against the oracle's exact int64
product, bit-exact, through the C ABI: every input format, ragged shapes that leave partial
tiles in M, N and K, the narrowest-width output and fixed (masking) output widths.  Slab
operands of one width take the fused path (operands unpacked in shared memory, the product
packed from the accumulators): every width 1..8, every output format, the repack when the
precomputed packing width overshoots, and byte equality with the two-pass path."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import NOGAPS, PLAIN32, PLAIN64, SLAB

pytestmark = pytest.mark.gpu


def matrix_upload(raw, n, fmt, bits):
    import torch

    from amethyst_b200.ops import PackedColumn, alloc_bytes

    buf = alloc_bytes(len(raw))
    buf[: len(raw)].copy_(torch.from_numpy(raw.copy()))
    return PackedColumn(buf, n, fmt, bits)


def dirty_slab_matrix(raw, bits, seed):
    """Random garbage in the dead top bits of every slab word (readers must ignore them)."""
    eps = 64 // bits
    live = eps * bits
    raw = raw.copy()
    if live < 64:
        w = raw[: len(raw) // 8 * 8].view(np.uint64)
        junk = np.random.default_rng(seed).integers(0, 2**63, size=w.size, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
        w |= junk & np.uint64(~((1 << live) - 1) & 0xFFFFFFFFFFFFFFFF)
    return raw


def check_case(m, n, k, af, ab, bf, bb, of, ob, seed, av=None, bv=None):
    from amethyst_b200 import ops

    av = O.uniform_values(seed, ab, m * k) if av is None else av
    bv = O.uniform_values(seed + 1, bb, k * n) if bv is None else bv
    araw = O.matrix_encode(af, ab, av, m, k)
    braw = O.matrix_encode(bf, bb, bv, k, n)
    if af == SLAB:
        araw = dirty_slab_matrix(araw, ab, seed + 2)
    if bf == SLAB:
        braw = dirty_slab_matrix(braw, bb, seed + 3)
    want = O.matmul(araw, af, ab, braw, bf, bb, m, n, k, threads=os.cpu_count() or 1).astype(np.uint64)
    mx = int(want.max()) if want.size else 0
    width = ob if ob else max(1, mx.bit_length())
    a = matrix_upload(araw, m * k, af, ab)
    b = matrix_upload(braw, k * n, bf, bb)
    out, wdev = ops.matmul(a, b, m, n, k, out_fmt=of, out_bits=ob)
    assert int(wdev[0].item()) == width
    exp = O.matrix_encode(of, width, want.reshape(-1) & np.uint64((1 << width) - 1), m, n)
    nb = int(O.ora().ora_matrix_words(of, width, m, n)) * (4 if of == PLAIN32 else 8)
    got = out.data[:nb].cpu().numpy()
    assert np.array_equal(got, exp[:nb]), (m, n, k, af, ab, bf, bb, of, ob)


CASES = [
    # M, N, K, a fmt, a bits, b fmt, b bits, out fmt, out bits
    (128, 256, 128, SLAB, 7, SLAB, 7, SLAB, 0),      # exactly one tile, one K slice
    (256, 512, 512, SLAB, 7, SLAB, 7, SLAB, 0),      # several tiles and K slices
    (100, 200, 300, SLAB, 7, SLAB, 5, PLAIN32, 0),   # partial tiles in M, N and K
    (1, 1, 1, PLAIN32, 8, PLAIN32, 8, PLAIN64, 0),
    (333, 517, 129, NOGAPS, 3, PLAIN64, 8, NOGAPS, 0),
    (129, 257, 1000, SLAB, 8, SLAB, 8, SLAB, 20),    # fixed narrower output: entries masked
    (77, 300, 64, PLAIN64, 1, NOGAPS, 2, PLAIN32, 32),
    (300, 300, 4096, SLAB, 7, SLAB, 7, SLAB, 0),     # the matrix configuration's K
    (640, 768, 896, SLAB, 6, SLAB, 8, NOGAPS, 0),
]


@pytest.mark.parametrize("m,n,k,af,ab,bf,bb,of,ob", CASES)
def test_matmul_matches_oracle(cuda, m, n, k, af, ab, bf, bb, of, ob):
    check_case(m, n, k, af, ab, bf, bb, of, ob, seed=m * 7 + n * 3 + k)


def test_matmul_degenerate_shapes(cuda):
    """K = 0 gives an all-zero product written at width 1; M = 0 writes nothing."""
    import torch

    from amethyst_b200 import ops

    a = matrix_upload(np.zeros(16, np.uint8), 0, SLAB, 7)
    b = matrix_upload(np.zeros(16, np.uint8), 0, SLAB, 7)
    out, w = ops.matmul(a, b, 64, 64, 0, out_fmt=SLAB, out_bits=0)
    torch.cuda.synchronize()
    assert int(w[0].item()) == 1
    nb = int(O.ora().ora_matrix_words(SLAB, 1, 64, 64)) * 8
    assert not out.data[:nb].any().item()
    out, w = ops.matmul(a, b, 0, 5, 0, out_fmt=PLAIN32, out_bits=0)
    assert int(w[0].item()) == 1


def test_matmul_rejects_overflowing_widths(cuda):
    """Entries wider than 8 bits, or K * max(a) * max(b) beyond int32, are refused by the C ABI."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    L = A.lib()
    ws = ops.matmul_workspace(64, 64, 64)
    out = ops.PackedColumn(ops.alloc_bytes(64 * 64 * 4), 64 * 64, PLAIN32, 32)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    a = matrix_upload(np.zeros(64 * 64 * 4, np.uint8), 64 * 64, PLAIN32, 9)
    b = matrix_upload(np.zeros(64 * 64 * 4, np.uint8), 64 * 64, PLAIN32, 8)
    st = L.amx_matmul(C.byref(a.desc), C.byref(b.desc), 64, 64, 64, C.byref(out.desc), None,
                      C.c_void_p(ws.data_ptr()), ws.numel(), s)
    assert st == 2  # AMX_ERR_UNSUPPORTED
    big = 40000  # 40000 * 255 * 255 > 2^31
    a = matrix_upload(np.zeros(16, np.uint8), big, PLAIN32, 8)
    b = matrix_upload(np.zeros(16, np.uint8), big, PLAIN32, 8)
    st = L.amx_matmul(C.byref(a.desc), C.byref(b.desc), 1, 1, big, C.byref(out.desc), None,
                      C.c_void_p(ws.data_ptr()), ws.numel(), s)
    assert st == 2


def test_matmul_repeated_and_status(cuda):
    """Two calls on one workspace give the same bytes and leave no device-side error."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    m, n, k = 384, 512, 1024
    av = O.uniform_values(5, 7, m * k)
    bv = O.uniform_values(6, 7, k * n)
    a = matrix_upload(O.matrix_encode(SLAB, 7, av, m, k), m * k, SLAB, 7)
    b = matrix_upload(O.matrix_encode(SLAB, 7, bv, k, n), k * n, SLAB, 7)
    ws = ops.matmul_workspace(m, n, k)
    o1, w1 = ops.matmul(a, b, m, n, k, ws=ws)
    r1 = o1.data.clone()
    o2, w2 = ops.matmul(a, b, m, n, k, ws=ws)
    torch.cuda.synchronize()
    assert torch.equal(r1, o2.data) and int(w1[0].item()) == int(w2[0].item())
    A.check(A.lib().amx_matmul_status(C.c_void_p(ws.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))


@pytest.fixture
def fused_policy(request):
    """amx_tuning.policy 2 (the fused kernel, packed stages by TMA where the row pitches allow)
    or 3 (the fused kernel reading the packed words from global memory) for the test."""
    import ctypes as C

    from amethyst_b200 import _capi as A

    A.check(A.lib().amx_set_tuning(C.byref(A.Tuning(0, 0, request.param, 0))))
    yield request.param
    A.check(A.lib().amx_set_tuning(None))


FUSED_CASES = [
    # M, N, K, bits (both operands, slabs), out fmt, out bits
    (128, 256, 128, 1, SLAB, 0),
    (200, 300, 500, 2, NOGAPS, 0),
    (129, 257, 385, 3, SLAB, 0),      # 21 fields per slab: every run residue, partial tiles
    (256, 512, 640, 4, PLAIN32, 0),
    (100, 1000, 300, 5, SLAB, 0),
    (333, 517, 1000, 6, NOGAPS, 0),
    (300, 600, 2048, 7, SLAB, 0),
    (257, 255, 129, 8, PLAIN64, 0),
    (128, 256, 256, 7, SLAB, 20),     # fixed narrower width: entries masked
    (130, 260, 200, 5, NOGAPS, 13),
    (64, 64, 64, 8, PLAIN32, 11),
    (100, 300, 128, 7, SLAB, 40),     # fixed width above 32: one entry per slab
    (1, 1, 1, 7, SLAB, 0),
    (520, 270, 4096, 7, NOGAPS, 0),   # the matrix configuration's K, tile edges inside words
    (384, 576, 1530, 7, SLAB, 0),     # even row pitches: packed stages by TMA
    (333, 517, 1000, 6, NOGAPS, 0),
    (256, 768, 1024, 3, PLAIN32, 0),
]


@pytest.mark.parametrize("fused_policy", [2, 3], indirect=True)
@pytest.mark.parametrize("m,n,k,bits,of,ob", FUSED_CASES)
def test_fused_matmul_matches_oracle(cuda, fused_policy, m, n, k, bits, of, ob):
    check_case(m, n, k, SLAB, bits, SLAB, bits, of, ob, seed=m * 5 + n * 11 + k + bits)


@pytest.mark.parametrize("fused_policy", [2], indirect=True)
def test_fused_repack_when_the_bound_overshoots(cuda, fused_policy):
    """A nonzero only in even columns and B's even rows only 0/1: the products stay small while
    the row and column norms (the packing-width bound) are large, so the output is packed wide
    and then repacked at the narrowest width.  Also the all-zero product (disjoint supports)."""
    m, n, k, bits = 200, 300, 1024, 7
    rng = np.random.default_rng(3)
    a = rng.integers(0, 128, size=(m, k), dtype=np.uint64)
    a[:, 1::2] = 0
    b = rng.integers(0, 128, size=(k, n), dtype=np.uint64)
    b[0::2, :] = rng.integers(0, 2, size=(k // 2, n), dtype=np.uint64)
    for of in (SLAB, NOGAPS):
        check_case(m, n, k, SLAB, bits, SLAB, bits, of, 0, seed=4, av=a.reshape(-1), bv=b.reshape(-1))
    b[0::2, :] = 0
    for of in (SLAB, NOGAPS, PLAIN32):
        check_case(m, n, k, SLAB, bits, SLAB, bits, of, 0, seed=5, av=a.reshape(-1), bv=b.reshape(-1))


def test_fused_and_two_pass_paths_agree(cuda):
    """The same product through the fused kernel (amx_tuning.policy = 2, packed stages by TMA:
    both row pitches are 170 and 72 words) and the default two-pass path is byte-identical, for a
    slab and a nogaps output (K = 1530: the packing-width bound is one bit above the final width,
    so the fused path also repacks here)."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    m, n, k = 384, 640, 1530
    a = matrix_upload(O.matrix_encode(SLAB, 7, O.uniform_values(11, 7, m * k), m, k), m * k, SLAB, 7)
    b = matrix_upload(O.matrix_encode(SLAB, 7, O.uniform_values(12, 7, k * n), k, n), k * n, SLAB, 7)
    try:
        for of in (SLAB, NOGAPS):
            o2, w2 = ops.matmul(a, b, m, n, k, out_fmt=of)
            A.check(A.lib().amx_set_tuning(C.byref(A.Tuning(0, 0, 2, 0))))
            o1, w1 = ops.matmul(a, b, m, n, k, out_fmt=of)
            A.check(A.lib().amx_set_tuning(None))
            torch.cuda.synchronize()
            width = int(w1[0].item())
            assert width == int(w2[0].item())
            nb = int(O.ora().ora_matrix_words(of, width, m, n)) * 8  # bytes past these are not output
            assert torch.equal(o1.data[:nb], o2.data[:nb]), of
    finally:
        A.check(A.lib().amx_set_tuning(None))
