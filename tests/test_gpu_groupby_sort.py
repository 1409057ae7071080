"""The sort-based group-by (amx_groupby_sort: LSD radix sort of the key/value pairs, then
reduce-by-key -- the reference's cub::DeviceRadixSort::SortPairs + ReduceByKey path) against the
oracle's sort + reduce-by-key group-by, bit-exact, through the C ABI: key widths 1..32 (one to
four digit passes), lengths around the 4096-pair tiles, runs that cross tiles, every pair its own
group, one group for everything, values wider than 32 bits, masks, and outputs too small."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import NOGAPS, PLAIN32, PLAIN64, SLAB, gpu_bytes, make_column, to_gpu
from tests.test_gpu_groupby import wide_keys, zipf_keys

pytestmark = pytest.mark.gpu

CASES = [
    # key fmt, key bits, val fmt, val bits, n, distinct keys (0: uniform over the key space)
    (SLAB, 32, SLAB, 16, 1 << 20, 100000),    # high cardinality, Zipf weights
    (PLAIN32, 32, PLAIN32, 20, 300001, 0),    # nearly every key distinct
    (SLAB, 10, SLAB, 16, 1 << 20, 1000),      # the group-by configuration's shape, reduced
    (SLAB, 1, SLAB, 5, 65537, 0),             # one pass, two keys
    (NOGAPS, 9, SLAB, 21, 123457, 0),         # two passes, the second of one bit
    (SLAB, 17, NOGAPS, 13, 400003, 0),        # three passes
    (PLAIN64, 24, PLAIN64, 40, 77777, 3000),  # values wider than 32 bits
    (SLAB, 32, PLAIN64, 64, 50001, 700),      # 64-bit values
    (SLAB, 28, SLAB, 7, 4095, 0),
    (SLAB, 28, SLAB, 7, 4096, 0),
    (SLAB, 28, SLAB, 7, 4097, 0),
    (SLAB, 30, SLAB, 30, 1, 0),
    (SLAB, 30, SLAB, 30, 0, 0),
]


def _check(kc, vc, kb, n, want, mask=None, key_fmt=PLAIN32, max_groups=None):
    from amethyst_b200 import ops

    g, wk, ws, wc = want
    ok, osum, ocnt, ng = ops.groupby_sort(kc, vc, key_fmt=key_fmt, mask=mask, max_groups=max_groups)
    assert int(ng[0].item()) == g
    kbits = kb if key_fmt == SLAB else 32
    assert np.array_equal(gpu_bytes(ok, g), O.encode(key_fmt, kbits, wk)[: O.storage_bytes(key_fmt, kbits, g)])
    assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), ws)
    assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), wc)


@pytest.mark.parametrize("kf,kb,vf,vb,n,distinct", CASES)
def test_groupby_sort_matches_the_sorting_oracle(cuda, kf, kb, vf, vb, n, distinct):
    keys = wide_keys(n, kb, distinct, kb * 3 + n) if n else np.zeros(0, np.uint64)
    kv, kraw = make_column(kb * 17 + n, kf, kb, n, vals=keys)
    vv, vraw = make_column(vb * 19 + n, vf, vb, n)
    kc, vc = to_gpu(kraw, n, kf, kb), to_gpu(vraw, n, vf, vb)
    want = O.groupby_sorted(kraw, kf, kb, vraw, vf, vb, n)
    for key_fmt in (PLAIN32, SLAB):
        _check(kc, vc, kb, n, want, key_fmt=key_fmt)


def test_groupby_sort_runs_across_tiles_and_single_group(cuda):
    """Sorted runs far longer than a tile (a few hot keys), and one key for every pair."""
    n, kb = 3 * 4096 * 7 + 11, 20
    rng = np.random.default_rng(8)
    keys = rng.choice(np.array([3, 77, (1 << kb) - 1, 1000], np.uint64), size=n, p=[0.6, 0.3, 0.09, 0.01])
    kv, kraw = make_column(1, SLAB, kb, n, vals=keys)
    vv, vraw = make_column(2, SLAB, 16, n)
    _check(to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16), kb, n,
           O.groupby_sorted(kraw, SLAB, kb, vraw, SLAB, 16, n))
    keys = np.full(n, 12345, np.uint64)
    kv, kraw = make_column(3, SLAB, kb, n, vals=keys)
    _check(to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16), kb, n,
           O.groupby_sorted(kraw, SLAB, kb, vraw, SLAB, 16, n))


def test_groupby_sort_with_mask_and_capacity(cuda):
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n, kb = 200003, 32
    keys = wide_keys(n, kb, 5000, 9)
    kv, kraw = make_column(91, SLAB, kb, n, vals=keys)
    vv, vraw = make_column(92, SLAB, 16, n)
    kc, vc = to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16)
    m = np.random.default_rng(5).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    m[-1] &= np.uint32((1 << (n % 32)) - 1)
    mask = torch.from_numpy(np.concatenate([m, np.zeros(4, np.uint32)]).view(np.int32)).cuda()
    _check(kc, vc, kb, n, O.groupby_sorted(kraw, SLAB, kb, vraw, SLAB, 16, n, mask=m), mask=mask)
    # more groups than the outputs hold: reported, never written past them
    ws = ops.aligned_bytes(int(A.lib().amx_groupby_sort_workspace_bytes(n, kb, 16)), 256)
    ok, osum, ocnt, ng = ops.groupby_sort(kc, vc, max_groups=1000, ws=ws)
    with pytest.raises(A.AmxError) as e:
        A.check(A.lib().amx_groupby_sort_status(C.c_void_p(ws.data_ptr()),
                                                C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert e.value.status == 7  # AMX_ERR_CAPACITY


def test_groupby_sort_agrees_with_the_hash_group_by(cuda):
    """The same groups from amx_groupby (dense table, hash table, wide-key hash table) and
    amx_groupby_sort."""
    import torch

    from amethyst_b200 import ops

    for kb, distinct in ((10, 1000), (20, 0), (32, 20000)):
        n = 300007
        keys = zipf_keys(n, 1 << kb, 1.1, kb) if kb <= 10 else wide_keys(n, kb, distinct, kb)
        kv, kraw = make_column(kb, SLAB, kb, n, vals=keys)
        vv, vraw = make_column(kb + 1, SLAB, 16, n)
        kc, vc = to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16)
        a = ops.groupby(kc, vc, max_groups=1 << 19)
        b = ops.groupby_sort(kc, vc)
        g = int(a[3][0].item())
        assert g == int(b[3][0].item())
        for x, y in zip(a[:3], b[:3]):
            nb = O.storage_bytes(x.fmt, x.bits, g)
            assert torch.equal(x.data[:nb], y.data[:nb])


def test_groupby_auto_picks_by_expected_groups(cuda):
    """ops.groupby_auto: the hash tables below n / 128 expected groups, the sort from there on;
    both give the oracle's groups."""
    from unittest import mock

    from amethyst_b200 import ops

    n, kb = 100003, 32
    keys = wide_keys(n, kb, 20000, 4)
    kv, kraw = make_column(41, SLAB, kb, n, vals=keys)
    vv, vraw = make_column(42, SLAB, 16, n)
    kc, vc = to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16)
    g, wk, ws, wc = O.groupby_sorted(kraw, SLAB, kb, vraw, SLAB, 16, n)
    for hint, expect_sort in ((100, False), (n // 128 + 1, True), (20000, True)):
        with mock.patch.object(ops, "groupby_sort", wraps=ops.groupby_sort) as gs:
            ok, osum, ocnt, ng = ops.groupby_auto(kc, vc, hint, max_groups=1 << 16)
        assert gs.called == expect_sort, hint
        assert int(ng[0].item()) == g
        assert np.array_equal(gpu_bytes(ok, g).view(np.uint32), wk.astype(np.uint32))
        assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), ws)
        assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), wc)
