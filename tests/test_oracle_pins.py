"""The C oracle against the reference's own host code run live (oracle/_ref/libamxref_host.so),
on fresh random inputs, plus the oracle's own algebraic consistency.  Skipped where the
reference could not be built (the GPU machine has no reference tree)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def ref():
    h = O.ref_host()
    if h is None:
        try:
            O.build(with_reference=True)
        except Exception:
            pass
        h = O.ref_host()
    if h is None:
        pytest.skip("reference host code not built (no reference tree)")
    return h


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_accessors_live(ref, seed):
    rng = np.random.default_rng(seed)
    words = rng.integers(0, 2**63, size=64, dtype=np.uint64) * np.uint64(2) + np.uint64(seed & 1)
    raw = np.concatenate([words, np.zeros(4, np.uint64)]).view(np.uint8)
    for b in range(1, 65):
        n_slab = 64 * (64 // b)
        vals = O.decode(raw, n_slab, O.SLAB, b)
        for i in rng.choice(n_slab, size=min(n_slab, 40), replace=False):
            assert vals[i] == ref.amxref_get_element(b, O._p(words), int(i))
        n_ng = (63 * 64) // b
        vals = O.decode(raw, n_ng, O.NOGAPS, b)
        for i in rng.choice(n_ng, size=min(n_ng, 40), replace=False):
            assert vals[i] == ref.amxref_get_elem_nogaps(b, O._p(words), int(i))
        vals = O.decode(raw, 64, O.PLAIN64, b)
        for i in range(0, 64, 5):
            assert vals[i] == ref.amxref_get_element_baseline(b, O._p(words), i)


def test_operators_live(ref):
    rng = np.random.default_rng(7)
    for _ in range(400):
        ob = int(rng.integers(1, 65))
        lb = int(rng.integers(1, 33))
        lv = int(rng.integers(1, 1 << lb))
        rv = int(rng.integers(1, 1 << lb))
        for op in (0, 2, 3, 4, 10, 11, 12):
            assert O.ora().ora_binop(op, lv, rv, ob) == ref.amxref_op(op, ob, lv, rv), (op, ob, lv, rv)


def test_main_inputs_and_masks_live(ref):
    n = 1 << 14
    ok, d1, d2 = O.run_reference_main(["-n", str(n), "--nv"], n)
    assert ok
    e1, e2 = O.reference_inputs(42, n)
    assert np.array_equal(d1, e1) and np.array_equal(d2, e2)
    ok, _, m = O.run_reference_main(["-n", str(n), "--nv", "-m", "2", "-s", "0.25"], n)
    assert np.array_equal(m.view(np.uint8)[: n // 8], O.mask_clusters(0.25, 8, n))


def test_encode_decode_roundtrip():
    for fmt in (O.PLAIN32, O.PLAIN64, O.SLAB, O.NOGAPS):
        for b in ([1, 5, 11, 17, 31, 32] + ([] if fmt == O.PLAIN32 else [33, 50, 63, 64])):
            for n in (0, 1, 63, 64, 65, 1000):
                v = O.uniform_values(b * 1000 + n, b, n)
                raw = O.encode(fmt, b, v)
                assert np.array_equal(O.decode(raw, n, fmt, b), v)


def test_compressstore_is_filter_then_select():
    n = 5000
    v = O.uniform_values(3, 11, n)
    raw = O.encode(O.SLAB, 11, v)
    p = O.pred(1, 205)
    mask = O.filter(raw, n, O.SLAB, 11, p)
    out1, c1 = O.compressstore(raw, n, O.SLAB, 11, mask, O.SLAB, 11)
    out2, c2 = O.filter_compressstore(raw, n, O.SLAB, 11, p, O.SLAB, 11)
    assert c1 == c2 == int((v < 205).sum())
    assert np.array_equal(out1, out2)
    assert np.array_equal(O.decode(out1, c1, O.SLAB, 11), v[v < 205])


def test_chain_compress_mt_matches_chain():
    """The multi-threaded chain with compacted output (the CPU baseline's routine) agrees with the
    single-threaded oracle chain on counts, aggregates and output bytes."""
    for n, threads in ((0, 3), (1, 4), (100003, 7), (65536, 1)):
        a, b = O.uniform_values(5, 7, n), O.uniform_values(6, 13, n)
        ar, br = O.encode(2, 7, a), O.encode(2, 13, b)
        for fmt, bits in ((2, 14), (0, 32), (3, 14)):
            p = O.pred(4, 4160)
            w = O.chain(0, (ar, 2, 7), (br, 2, 13), 14, p, 0, fmt, bits, n)
            g = O.chain_compress_mt(0, (ar, 2, 7), (br, 2, 13), 14, p, 0, fmt, bits, n, threads)
            assert w[1:] == g[1:] and np.array_equal(w[0], g[0])


def test_sorted_groupby_matches_dense_groupby():
    """The oracle's sort + reduce-by-key group-by (wide keys) agrees with its dense-table group-by
    wherever the dense table fits, with and without a mask."""
    for n, kb, vb in ((0, 5, 5), (1, 3, 9), (20011, 10, 16), (50000, 16, 33)):
        k = O.uniform_values(kb + n, kb, n)
        v = O.uniform_values(vb + n + 1, vb, n)
        kr, vr = O.encode(2, kb, k), O.encode(3, vb, v)
        g1, s1, c1 = O.groupby_dense(kr, 2, kb, vr, 3, vb, n)
        g2, k2, s2, c2 = O.groupby_sorted(kr, 2, kb, vr, 3, vb, n)
        pres = np.nonzero(c1)[0]
        assert g1 == g2 and np.array_equal(k2, pres) and np.array_equal(s2, s1[pres]) and np.array_equal(c2, c1[pres])
        if n:
            m = np.random.default_rng(n).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
            g3, k3, s3, c3 = O.groupby_sorted(kr, 2, kb, vr, 3, vb, n, mask=m)
            bits = np.unpackbits(m.view(np.uint8), bitorder="little")[:n].astype(bool)
            kk, vv = k[bits], v[bits]
            uk = np.unique(kk)
            assert g3 == len(uk) and np.array_equal(k3, uk)
            assert np.array_equal(c3, np.array([np.sum(kk == u) for u in uk[:50]] + list(c3[50:]), dtype=np.uint64))
