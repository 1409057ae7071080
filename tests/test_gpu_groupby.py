"""Group-by sum + count against the oracle's dense group table, bit-exact, through the C ABI."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import NOGAPS, PLAIN32, PLAIN64, SLAB, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu


def zipf_keys(n, groups, s, seed):
    from amethyst_b200.datagen import zipf_cdf

    cdf = zipf_cdf(groups, s)
    u = np.random.default_rng(seed).random(n)
    return np.searchsorted(cdf, u, side="right").astype(np.uint64)


CASES = [
    # key fmt, key bits, val fmt, val bits, n, key distribution
    (SLAB, 10, SLAB, 16, 1 << 20, "zipf"),      # the group-by configuration at reduced size
    (SLAB, 10, SLAB, 10, 300001, "zipf"),       # the reference's layout: keys and values share b
    (PLAIN32, 12, PLAIN32, 32, 200003, "uniform"),
    (NOGAPS, 7, NOGAPS, 13, 123457, "uniform"),
    (SLAB, 16, SLAB, 16, 500000, "zipf"),       # hash path
    (SLAB, 20, PLAIN32, 20, 400001, "uniform"),  # hash path with spills
    (PLAIN64, 24, SLAB, 7, 100000, "uniform"),
    (SLAB, 11, PLAIN64, 40, 77777, "zipf"),     # values wider than 32 bits
    (SLAB, 3, SLAB, 5, 4096, "uniform"),
    (SLAB, 5, SLAB, 5, 0, "uniform"),
    (SLAB, 5, SLAB, 5, 1, "uniform"),
]


@pytest.mark.parametrize("kf,kb,vf,vb,n,dist", CASES)
def test_groupby_matches_oracle(cuda, kf, kb, vf, vb, n, dist):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    keys = zipf_keys(n, min(1000, 1 << kb), 1.1, kb * 7 + n) if dist == "zipf" else None
    kv, kraw = make_column(kb * 101 + n, kf, kb, n, vals=keys)
    vv, vraw = make_column(vb * 103 + n, vf, vb, n)
    kc, vc = to_gpu(kraw, n, kf, kb), to_gpu(vraw, n, vf, vb)
    groups, sums, counts = O.groupby_dense(kraw, kf, kb, vraw, vf, vb, n)
    present = np.nonzero(counts)[0].astype(np.uint64)
    for sum_fmt, sum_bits in [(PLAIN64, 64), (SLAB, kb)]:
        ok, osum, ocnt, ng = ops.groupby(kc, vc, key_fmt=SLAB, sum_fmt=sum_fmt, sum_bits=sum_bits,
                                         count_fmt=PLAIN64)
        g = int(ng[0].item())
        assert g == groups
        assert np.array_equal(gpu_bytes(ok, g), O.encode(SLAB, kb, present)[: O.storage_bytes(SLAB, kb, g)])
        assert np.array_equal(gpu_bytes(osum, g),
                              O.encode(sum_fmt, sum_bits, sums[present.astype(np.int64)])[
                                  : O.storage_bytes(sum_fmt, sum_bits, g)])
        assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), counts[present.astype(np.int64)])


def test_groupby_with_mask(cuda):
    import torch

    from amethyst_b200 import ops

    n = 250001
    keys = zipf_keys(n, 1000, 1.1, 3)
    kv, kraw = make_column(1, SLAB, 10, n, vals=keys)
    vv, vraw = make_column(2, SLAB, 16, n)
    m = np.random.default_rng(4).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    m[-1] &= np.uint32((1 << (n % 32)) - 1)
    dm = torch.zeros(len(m) + 4, dtype=torch.int32, device="cuda")
    dm[: len(m)].copy_(torch.from_numpy(m.view(np.int32)))
    sel = np.unpackbits(m.view(np.uint8), bitorder="little")[:n].astype(bool)
    want_sum = np.zeros(1024, np.uint64)
    want_cnt = np.zeros(1024, np.uint64)
    np.add.at(want_sum, kv[sel].astype(np.int64), vv[sel])
    np.add.at(want_cnt, kv[sel].astype(np.int64), 1)
    ok, osum, ocnt, ng = ops.groupby(to_gpu(kraw, n, SLAB, 10), to_gpu(vraw, n, SLAB, 16), key_fmt=PLAIN32, mask=dm)
    present = np.nonzero(want_cnt)[0]
    g = int(ng[0].item())
    assert g == len(present)
    assert np.array_equal(gpu_bytes(ok, g).view(np.uint32), present.astype(np.uint32))
    assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), want_sum[present])
    assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), want_cnt[present])


@pytest.mark.parametrize("kf,kb,vf,vb", [
    (SLAB, 10, SLAB, 16),     # dense table without carry words: flushed every 2^16 elements
    (SLAB, 16, SLAB, 18),     # hash table without carry words: flushed every chunk (2^14)
    (SLAB, 10, PLAIN32, 32),  # dense table, 32-bit sums with carry words
    (NOGAPS, 9, SLAB, 21),    # general key reader, carry words
    (PLAIN32, 12, NOGAPS, 3),  # general readers on both columns
])
def test_groupby_one_cta_flushes(cuda, kf, kb, vf, vb):
    """One CTA aggregates 2^20 + 12345 elements, so its shared table is flushed mid-column
    whenever a carry-free 32-bit sum could otherwise wrap: values at the top of their range on
    one hot key reach the largest sums and counts the shared fields must hold."""
    import ctypes as C

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = (1 << 20) + 12345
    rng = np.random.default_rng(kb * 1000 + vb)
    keys = rng.integers(0, 1 << kb, size=n, dtype=np.uint64)
    keys[rng.random(n) < 0.8] = 5
    vals = np.full(n, (1 << vb) - 1, np.uint64)
    low = rng.random(n) < 0.1
    vals[low] = rng.integers(0, 1 << vb, size=int(low.sum()), dtype=np.uint64)
    kv, kraw = make_column(1, kf, kb, n, vals=keys)
    vv, vraw = make_column(2, vf, vb, n, vals=vals)
    want_sum = np.zeros(1 << kb, np.uint64)
    want_cnt = np.zeros(1 << kb, np.uint64)
    np.add.at(want_sum, kv.astype(np.int64), vv)
    np.add.at(want_cnt, kv.astype(np.int64), 1)
    t = A.Tuning(0, 0, 0, 1)
    A.check(A.lib().amx_set_tuning(C.byref(t)))
    try:
        ok, osum, ocnt, ng = ops.groupby(to_gpu(kraw, n, kf, kb), to_gpu(vraw, n, vf, vb), key_fmt=PLAIN32)
        g = int(ng[0].item())
    finally:
        A.check(A.lib().amx_set_tuning(None))
    present = np.nonzero(want_cnt)[0]
    assert want_cnt[5] > (1 << 19)
    assert g == len(present)
    assert np.array_equal(gpu_bytes(ok, g).view(np.uint32), present.astype(np.uint32))
    assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), want_sum[present])
    assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), want_cnt[present])


WIDE_CASES = [
    # key fmt, key bits, val fmt, val bits, n, distinct keys (0: uniform over the key space)
    (SLAB, 32, SLAB, 16, 1 << 20, 1000),       # Zipf-weighted draws from 1000 random 32-bit keys
    (PLAIN32, 32, PLAIN32, 20, 300001, 0),     # nearly every key distinct: ~300K groups
    (PLAIN32, 32, SLAB, 16, 1 << 20, 0),       # ~2^20 distinct groups
    (SLAB, 25, NOGAPS, 13, 400003, 0),         # ~4K collisions in a 25-bit space
    (NOGAPS, 28, SLAB, 7, 123457, 50000),
    (PLAIN64, 32, PLAIN64, 40, 77777, 3000),   # values wider than 32 bits
    (SLAB, 30, SLAB, 30, 1, 0),
    (SLAB, 30, SLAB, 30, 0, 0),
]


def wide_keys(n, bits, distinct, seed):
    rng = np.random.default_rng(seed)
    if distinct == 0:
        k = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    else:
        pool = rng.choice(1 << bits, size=distinct, replace=False).astype(np.uint64)
        pool[0] = (1 << bits) - 1  # the all-ones key too
        k = pool[zipf_keys(n, distinct, 1.1, seed + 1).astype(np.int64)]
    return k


@pytest.mark.parametrize("kf,kb,vf,vb,n,distinct", WIDE_CASES)
def test_groupby_wide_keys_match_the_sorting_oracle(cuda, kf, kb, vf, vb, n, distinct):
    """Keys of 25..32 bits: global hash table, groups in ascending key order, against the oracle's
    sort + reduce-by-key group-by (the reference's sort-based path)."""
    from amethyst_b200 import ops

    keys = wide_keys(n, kb, distinct, kb + n)
    kv, kraw = make_column(kb * 11 + n, kf, kb, n, vals=keys)
    vv, vraw = make_column(vb * 13 + n, vf, vb, n)
    kc, vc = to_gpu(kraw, n, kf, kb), to_gpu(vraw, n, vf, vb)
    g, wk, ws, wc = O.groupby_sorted(kraw, kf, kb, vraw, vf, vb, n)
    cap = max(1024, 2 * g)
    for key_fmt in (PLAIN32, SLAB):
        ok, osum, ocnt, ng = ops.groupby(kc, vc, key_fmt=key_fmt, max_groups=cap)
        gg = int(ng[0].item())
        assert gg == g
        assert np.array_equal(gpu_bytes(ok, g), O.encode(key_fmt, kb if key_fmt == SLAB else 32, wk)[
            : O.storage_bytes(key_fmt, kb if key_fmt == SLAB else 32, g)])
        assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), ws)
        assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), wc)


def test_groupby_wide_keys_with_mask_and_capacity(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n, kb = 200003, 32
    keys = wide_keys(n, kb, 5000, 9)
    kv, kraw = make_column(91, SLAB, kb, n, vals=keys)
    vv, vraw = make_column(92, SLAB, 16, n)
    kc, vc = to_gpu(kraw, n, SLAB, kb), to_gpu(vraw, n, SLAB, 16)
    m = np.random.default_rng(5).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    mask = torch.from_numpy(np.concatenate([m, np.zeros(4, np.uint32)]).view(np.int32)).cuda()
    g, wk, ws, wc = O.groupby_sorted(kraw, SLAB, kb, vraw, SLAB, 16, n, mask=m)
    wsp = ops.groupby_workspace(kb, 8192)
    ok, osum, ocnt, ng = ops.groupby(kc, vc, mask=mask, max_groups=8192, ws=wsp)
    ops.groupby_status(wsp, kb)
    assert int(ng[0].item()) == g
    assert np.array_equal(gpu_bytes(ok, g).view(np.uint32), wk.astype(np.uint32))
    assert np.array_equal(gpu_bytes(osum, g).view(np.uint64), ws)
    assert np.array_equal(gpu_bytes(ocnt, g).view(np.uint64), wc)
    # more distinct keys than the outputs hold: reported, never written past them
    small = ops.groupby_workspace(kb, 1024)
    ok2, osum2, ocnt2, ng2 = ops.groupby(kc, vc, max_groups=1024, ws=small)
    with pytest.raises(A.AmxError) as e:
        ops.groupby_status(small, kb)
    assert e.value.status == 7
