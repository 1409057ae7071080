"""Parity with the reference's OWN kernels, run on the same B200 on the same inputs: the
reference's src/kernels/*.cuh and CUB call sequences, compiled for sm_100a from the reference tree
into oracle/_ref/libamxref_gpu.so (test infrastructure, see oracle/ref_gpu.cu), against the C ABI
of this library.  Cases are the ones the reference's templates can express: filter with its
compiled-in predicate (v >= 2^(b-1)) and with v < 205, compressstore of slabs at the input width,
same-width binary ops (add at b+1 bits, mul at 2b bits), sums, the CUB plain paths, and the
shared-memory group-by (keys and values of one width, sums masked to that width).  Outputs are
compared as element values: the reference leaves some tail bits of its outputs untouched."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import PLAIN64, SLAB, make_column

pytestmark = pytest.mark.gpu

PAD = 1 << 20  # every device buffer the reference kernels touch gets 1 MiB of zeroed slack
GRID = 1024


@pytest.fixture(scope="module")
def ref():
    h = O.ref_gpu()
    if h is None:
        pytest.skip("reference kernels not built (oracle/_ref/libamxref_gpu.so)")
    return h


def dev(raw_or_nbytes):
    import torch

    if isinstance(raw_or_nbytes, int):
        return torch.zeros(raw_or_nbytes + PAD, dtype=torch.uint8, device="cuda")
    t = torch.zeros(len(raw_or_nbytes) + PAD, dtype=torch.uint8, device="cuda")
    t[: len(raw_or_nbytes)].copy_(torch.from_numpy(raw_or_nbytes.copy()))
    return t


def ptr(t):
    import ctypes as C

    return C.c_void_p(t.data_ptr())


def col(t, n, fmt, bits):
    from amethyst_b200.ops import PackedColumn

    return PackedColumn(t, n, fmt, bits)


SIZES = [1 << 16, 100000, 1 << 20]
WIDTHS = [3, 7, 11, 13, 16, 21, 32]


@pytest.mark.parametrize("bits", WIDTHS)
@pytest.mark.parametrize("n", SIZES)
def test_filter_and_compressstore_match_reference(cuda, ref, bits, n):
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    v, raw = make_column(bits * 977 + n, SLAB, bits, n)
    d = dev(raw)
    c = col(d, n, SLAB, bits)
    words = (n + 31) // 32
    for pred_id, p in [(0, ops.predicate(A.PRED_HALF, 0, 0, bits)), (1, ops.predicate(A.PRED_LT, 205, 0, bits))]:
        rmask = dev(8 * ((n + 63) // 64))
        assert ref.amxref_gpu_filter_slabs(bits, pred_id, ptr(d), n, ptr(rmask), GRID) == 0
        ours = ops.filter(c, p)
        torch.cuda.synchronize()
        assert np.array_equal(ours.cpu().numpy().view(np.uint32)[:words],
                              rmask[: 4 * words].cpu().numpy().view(np.uint32)), ("filter", bits, n, pred_id)
        # compressstore of the same mask: the reference's popcount -> CUB scan -> write pipeline
        rout = dev(O.storage_bytes(SLAB, bits, n))
        cnt = C.c_uint64(0)
        assert ref.amxref_gpu_compressstore_slabs(bits, ptr(rmask), ptr(d), ptr(rout), n, C.byref(cnt), GRID) == 0
        out, ocnt = ops.compressstore(c, ours, SLAB, bits)
        k = int(ocnt[0].item())
        assert k == cnt.value, ("count", bits, n, pred_id)
        got = O.decode(out.data[: O.storage_bytes(SLAB, bits, k)].cpu().numpy(), k, SLAB, bits)
        want = O.decode(rout[: O.storage_bytes(SLAB, bits, k)].cpu().numpy(), k, SLAB, bits)
        assert np.array_equal(got, want), ("compressstore", bits, n, pred_id)


@pytest.mark.parametrize("bits", [3, 7, 11, 13, 16, 21, 31])
def test_binary_ops_and_sum_match_reference(cuda, ref, bits):
    import ctypes as C

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 300007
    _, lraw = make_column(bits * 31 + 1, SLAB, bits, n)
    _, rraw = make_column(bits * 31 + 2, SLAB, bits, n)
    dl, dr = dev(lraw), dev(rraw)
    for op_id, op, ob in [(0, A.OP_ADD, bits + 1), (1, A.OP_MUL, 2 * bits)]:
        if ob > 64:
            continue
        rout = dev(O.storage_bytes(SLAB, ob, n))
        assert ref.amxref_gpu_binary_op_slabs(op_id, bits, ptr(dl), ptr(dr), ptr(rout), n, GRID) == 0
        ours = ops.binary_op(op, col(dl, n, SLAB, bits), col(dr, n, SLAB, bits), SLAB, ob)
        got = O.decode(ours.data[: O.storage_bytes(SLAB, ob, n)].cpu().numpy(), n, SLAB, ob)
        want = O.decode(rout[: O.storage_bytes(SLAB, ob, n)].cpu().numpy(), n, SLAB, ob)
        assert np.array_equal(got, want), ("binary", op_id, bits)
    s = C.c_uint64(0)
    assert ref.amxref_gpu_hop_slabs(bits, ptr(dl), n, C.byref(s), GRID) == 0
    ours = int(ops.hop(A.AGG_SUM, col(dl, n, SLAB, bits)).cpu().numpy().view(np.uint64)[0])
    assert ours == s.value


def test_cub_plain_paths_match_reference(cuda, ref):
    """cub::DeviceSelect::Flagged over the bit_iterator and cub::DeviceReduce over plain uint64
    words (the reference's baseline benches) against the plain64 format at 64 bits."""
    import ctypes as C

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 500003
    v, raw = make_column(5, PLAIN64, 64, n)
    d = dev(raw)
    m = np.random.default_rng(2).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    m[-1] &= np.uint32((1 << (n % 32)) - 1)
    dm = dev(m.view(np.uint8))
    rout = dev(8 * n)
    cnt = C.c_uint64(0)
    assert ref.amxref_gpu_compressstore_cub(ptr(dm), ptr(d), ptr(rout), n, C.byref(cnt)) == 0
    out, ocnt = ops.compressstore(col(d, n, PLAIN64, 64), dm, PLAIN64, 64)
    k = int(ocnt[0].item())
    assert k == cnt.value
    assert np.array_equal(out.data[: 8 * k].cpu().numpy(), rout[: 8 * k].cpu().numpy())
    s = C.c_uint64(0)
    assert ref.amxref_gpu_hop_cub(ptr(d), n, C.byref(s)) == 0
    assert int(ops.hop(A.AGG_SUM, col(d, n, PLAIN64, 64)).cpu().numpy().view(np.uint64)[0]) == s.value


@pytest.mark.parametrize("bits", [4, 7, 10, 12])
def test_groupby_matches_reference(cuda, ref, bits):
    """kernel_groupby_sm_array: keys and values share the width, aggregates masked to it, output
    order nondeterministic -- compared as sets of (key, aggregate) pairs."""
    import ctypes as C

    from amethyst_b200 import ops

    n = 200003
    _, kraw = make_column(bits * 13 + 1, SLAB, bits, n)
    _, vraw = make_column(bits * 13 + 2, SLAB, bits, n)
    dk, dv = dev(kraw), dev(vraw)
    g = 1 << bits
    rk, ra = dev(O.storage_bytes(SLAB, bits, g)), dev(O.storage_bytes(SLAB, bits, g))
    cnt = C.c_uint64(0)
    assert ref.amxref_gpu_groupby_sm_array(bits, ptr(dk), ptr(dv), ptr(rk), ptr(ra), n, C.byref(cnt), GRID) == 0
    k = cnt.value
    rkeys = O.decode(rk[: O.storage_bytes(SLAB, bits, k)].cpu().numpy(), k, SLAB, bits)
    raggs = O.decode(ra[: O.storage_bytes(SLAB, bits, k)].cpu().numpy(), k, SLAB, bits)
    ok, osum, ocnt, ng = ops.groupby(col(dk, n, SLAB, bits), col(dv, n, SLAB, bits), key_fmt=SLAB, sum_fmt=SLAB,
                                     sum_bits=bits)
    gcount = int(ng[0].item())
    assert gcount == k
    okeys = O.decode(ok.data[: O.storage_bytes(SLAB, bits, gcount)].cpu().numpy(), gcount, SLAB, bits)
    osums = O.decode(osum.data[: O.storage_bytes(SLAB, bits, gcount)].cpu().numpy(), gcount, SLAB, bits)
    assert sorted(zip(rkeys.tolist(), raggs.tolist())) == sorted(zip(okeys.tolist(), osums.tolist()))
