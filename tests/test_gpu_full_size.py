"""Every benchmark configuration at its full size, checked bit-exactly against the C oracle:
  - the 2^24-element filter + compressstore (also against the reference's own kernels);
  - the 1 GiB column (671,088,640 elements of 11 bits), encoded on the host by the oracle: the
    compacted bytes and the count against the oracle's filter + compressstore, whole buffer;
    plus properties with plain torch integer ops as an independent side (encode -> decode round
    trip of the device encoder, masked_select, bitmask popcount, count-only chain, sum);
  - the 2^26-element operator chain (and, through torch, its {packed, plain} x {packed, plain}
    forms);
  - the 2^28-element group-by against the oracle's dense-array group-by (and torch
    index_add_ / bincount);
  - the 4096^3 u7 matrix product: a 256-row block against the oracle's exact int64 product, the
    whole product against an fp64 product (exact below 2^53), and the narrowest output width;
  - 512 uneven columns in one batch: per-column count, sum and decoded output."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import PLAIN32, SLAB

pytestmark = pytest.mark.gpu

_POPC8 = None


def popcount_words(t):
    """Set bits of an int32 device tensor (a byte lookup table)."""
    import torch

    global _POPC8
    if _POPC8 is None or _POPC8.device != t.device:
        _POPC8 = torch.tensor([bin(i).count("1") for i in range(256)], dtype=torch.int64, device=t.device)
    return int(_POPC8[t.contiguous().view(torch.uint8).long()].sum().item())


def plain_col(vals, n):
    from amethyst_b200 import ops

    return ops.PackedColumn(vals.view(__import__("torch").uint8), n, PLAIN32, 32)


def values(n, bits, seed):
    """n uniform values below 2^bits, generated on the GPU (an int32 tensor: callers widen it to
    int64 and mask 32-bit values to their unsigned range)."""
    from amethyst_b200 import datagen

    return datagen.uniform_gpu(n, bits, seed)[:n]


def decoded(col, n):
    """The first n elements of a packed column as int64 (decoded by amx_convert to plain32)."""
    import torch

    from amethyst_b200 import ops

    if n == 0:
        return torch.zeros(0, dtype=torch.int64, device="cuda")
    src = ops.PackedColumn(col.data, n, col.fmt, col.bits)
    out = ops.convert(src, PLAIN32, 32)
    return out.data[: 4 * n].view(torch.int32).long() & 0xFFFFFFFF


def test_cfg1_filter_compressstore_vs_oracle(cuda):
    """2^24 elements at 11 bits, v < 205, 11-bit slabs out: bit-exact against the oracle and,
    when it is built, against the reference's popcount -> scan -> write kernels."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 1 << 24
    col = ops.convert(plain_col(values(n, 11, 0xCF61), n), SLAB, 11)
    raw = col.data[: col.nbytes].cpu().numpy()
    out, cnt = ops.filter_compressstore(col, ops.predicate(A.PRED_LT, 205, 0, 11), SLAB, 11)
    want, wcnt = O.filter_compressstore(raw, n, SLAB, 11, O.pred(A.PRED_LT, 205, 0, 11), SLAB, 11)
    got_n = int(cnt[0].item())
    assert got_n == wcnt and 0.09 < wcnt / n < 0.11
    nb = O.storage_bytes(SLAB, 11, wcnt)
    assert np.array_equal(out.data[:nb].cpu().numpy(), want[:nb])
    ref = O.ref_gpu()
    if ref is not None:
        pad = 1 << 20
        m8 = np.packbits((O.decode(raw, n, SLAB, 11) < 205).astype(np.uint8), bitorder="little")
        d = torch.zeros(len(raw) + pad, dtype=torch.uint8, device="cuda")
        d[: len(raw)].copy_(torch.from_numpy(raw.copy()))
        rm = torch.zeros(len(m8) + pad, dtype=torch.uint8, device="cuda")
        rm[: len(m8)].copy_(torch.from_numpy(m8))
        rout = torch.zeros(len(raw) + pad, dtype=torch.uint8, device="cuda")
        rc = C.c_uint64(0)
        assert ref.amxref_gpu_compressstore_slabs(11, C.c_void_p(rm.data_ptr()), C.c_void_p(d.data_ptr()),
                                                  C.c_void_p(rout.data_ptr()), n, C.byref(rc), 1024) == 0
        assert rc.value == wcnt
        assert np.array_equal(O.decode(rout[:nb].cpu().numpy(), wcnt, SLAB, 11), O.decode(want[:nb], wcnt, SLAB, 11))


def test_one_gib_column_vs_oracle(cuda):
    """The north-star column encoded on the host by the oracle (not by the device encoder),
    filtered v < 205 and compressstored on the GPU: the whole compacted buffer and the count
    against the oracle.  At 671,088,640 elements this covers the 64-bit index paths."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import datagen, ops

    n = (1 << 27) * 5
    raw = O.encode(SLAB, 11, datagen.uniform_np(0xC0FFEE, 11, n))
    nb = O.storage_bytes(SLAB, 11, n)
    assert nb == 1 << 30
    col = ops.PackedColumn.empty(n, SLAB, 11)
    col.data[:nb].copy_(torch.from_numpy(raw[:nb]))
    out, cnt = ops.filter_compressstore(col, ops.predicate(A.PRED_LT, 205, 0, 11), SLAB, 11)
    want, wcnt = O.filter_compressstore(raw, n, SLAB, 11, O.pred(A.PRED_LT, 205), SLAB, 11)
    del raw
    assert int(cnt[0].item()) == wcnt
    ob = O.storage_bytes(SLAB, 11, wcnt)
    assert np.array_equal(out.data[:ob].cpu().numpy(), want[:ob])


def test_one_gib_column_properties(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = (1 << 27) * 5  # 2^27 slabs of five 11-bit fields: 1 GiB
    v = values(n, 11, 0xC0FFEE)
    col = ops.convert(plain_col(v, n), SLAB, 11)
    assert col.nbytes == 1 << 30
    v = v.long()
    assert torch.equal(decoded(col, n), v)  # encode -> decode round trip
    p = ops.predicate(A.PRED_LT, 205, 0, 11)
    out, cnt = ops.filter_compressstore(col, p, SLAB, 11)
    c = int(cnt[0].item())
    keep = v < 205
    want = torch.masked_select(v, keep)
    del keep
    assert c == want.numel()
    assert torch.equal(decoded(out, c), want)
    del out
    torch.cuda.empty_cache()
    mask = ops.filter(col, p)
    assert popcount_words(mask[: (n + 31) // 32]) == c
    del mask
    _, _, ccnt, csum = ops.chain(col, None, A.OP_LHS, 11, p, A.AGG_SUM)
    assert int(ccnt[0].item()) == c
    assert int(csum[0].item()) == int(want.sum().item())


@pytest.mark.parametrize("in_plain", [False, True])
@pytest.mark.parametrize("out_plain", [False, True])
def test_chain_full_size(cuda, in_plain, out_plain):
    """A 2^26 x u7 + B 2^26 x u13 -> C at 14 bits, keep C >= 2^13, compressstore, sum, over
    packed or plain32 inputs into packed or plain32 output; packed -> packed also bit-exact
    against the oracle."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 1 << 26
    a, b = values(n, 7, 0x5EEDA), values(n, 13, 0x5EEDB)
    if in_plain:
        ca, cb = plain_col(a, n), plain_col(b, n)
    else:
        ca, cb = ops.convert(plain_col(a, n), SLAB, 7), ops.convert(plain_col(b, n), SLAB, 13)
    of, ob = (PLAIN32, 32) if out_plain else (SLAB, 14)
    p = ops.predicate(A.PRED_GE, 1 << 13, 0, 14)
    out, _, cnt, agg = ops.chain(ca, cb, A.OP_ADD, 14, p, A.AGG_SUM, out_fmt=of, out_bits=ob)
    s = a.long() + b.long()
    want = torch.masked_select(s, s >= (1 << 13))
    c = int(cnt[0].item())
    assert c == want.numel()
    assert int(agg[0].item()) == int(want.sum().item())
    assert torch.equal(decoded(out, c), want)
    if not in_plain and not out_plain:
        ra = ca.data[: ca.nbytes].cpu().numpy()
        rb = cb.data[: cb.nbytes].cpu().numpy()
        wout, wcnt, wagg = O.chain(A.OP_ADD, (ra, SLAB, 7), (rb, SLAB, 13), 14, O.pred(A.PRED_GE, 1 << 13, 0, 14),
                                   A.AGG_SUM, SLAB, 14, n)
        assert (c, int(agg[0].item())) == (wcnt, wagg)
        nb = O.storage_bytes(SLAB, 14, wcnt)
        assert np.array_equal(out.data[:nb].cpu().numpy(), wout[:nb])


def test_groupby_full_size(cuda):
    """2^28 Zipf(1.1) keys over 1000 groups at 10 bits, 2^28 u16 values at 16 bits."""
    import torch

    from amethyst_b200 import datagen, ops

    n = 1 << 28
    keys32, _ = datagen.keys_from_cdf_gpu(n, datagen.zipf_cdf(1000, 1.1), 0x21F)
    keys32 = keys32[:n]
    vals32 = values(n, 16, 0x7A1)
    keys = ops.convert(plain_col(keys32, n), SLAB, 10)
    vals = ops.convert(plain_col(vals32, n), SLAB, 16)
    ok, osum, ocnt, ng = ops.groupby(keys, vals)
    k = keys32.long()
    want_cnt = torch.bincount(k, minlength=1024)
    want_sum = torch.zeros(1024, dtype=torch.int64, device="cuda").index_add_(0, k, vals32.long())
    del k
    present = torch.nonzero(want_cnt).flatten()
    g = int(ng[0].item())
    assert g == present.numel()
    assert int(want_cnt.sum().item()) == n
    assert torch.equal(ok.data[: 4 * g].view(torch.int32).long(), present)
    assert torch.equal(osum.data[: 8 * g].view(torch.int64), want_sum[present])
    assert torch.equal(ocnt.data[: 8 * g].view(torch.int64), want_cnt[present])
    # the oracle's dense-array group-by over the same packed bytes
    kraw = keys.data[: keys.nbytes].cpu().numpy()
    vraw = vals.data[: vals.nbytes].cpu().numpy()
    og, osums, ocounts = O.groupby_dense(kraw, SLAB, 10, vraw, SLAB, 16, n)
    opresent = np.nonzero(ocounts)[0]
    assert og == g
    assert np.array_equal(ok.data[: 4 * g].view(torch.int32).cpu().numpy(), opresent.astype(np.int32))
    assert np.array_equal(osum.data[: 8 * g].cpu().numpy().view(np.uint64), osums[opresent])
    assert np.array_equal(ocnt.data[: 8 * g].cpu().numpy().view(np.uint64), ocounts[opresent])


def test_matmul_full_size(cuda):
    """4096^3 u7 x u7 slab matrices: int32 output against an fp64 product (every entry is below
    4096 * 127^2 < 2^53, so fp64 is exact), a row block against the oracle, the narrowest slab
    width of the output, and the fused kernel against both."""
    import torch

    from amethyst_b200 import ops

    m = n = k = 4096
    av = O.uniform_values(0xA7, 7, m * k)
    bv = O.uniform_values(0xB7, 7, k * n)
    araw = O.matrix_encode(SLAB, 7, av, m, k)
    braw = O.matrix_encode(SLAB, 7, bv, k, n)
    a = ops.PackedColumn(ops.alloc_bytes(len(araw)), m * k, SLAB, 7)  # rows padded to whole slabs
    a.data[: len(araw)].copy_(torch.from_numpy(araw))
    b = ops.PackedColumn(ops.alloc_bytes(len(braw)), k * n, SLAB, 7)
    b.data[: len(braw)].copy_(torch.from_numpy(braw))
    out, width = ops.matmul(a, b, m, n, k, out_fmt=PLAIN32, out_bits=32)
    ta = torch.from_numpy(av.astype(np.float64).reshape(m, k)).cuda()
    tb = torch.from_numpy(bv.astype(np.float64).reshape(k, n)).cuda()
    want = torch.matmul(ta, tb).long()
    got = out.data[: 4 * m * n].view(torch.int32).long().reshape(m, n)
    assert torch.equal(got, want)
    # rows 1024..1279 against the oracle's exact int64 product
    r0, rows = 1024, 256
    ablk = O.matrix_encode(SLAB, 7, av[r0 * k:(r0 + rows) * k], rows, k)
    oc = O.matmul(ablk, SLAB, 7, braw, SLAB, 7, rows, n, k, threads=os.cpu_count() or 1)
    assert np.array_equal(got[r0:r0 + rows].cpu().numpy(), oc)
    o2, w = ops.matmul(a, b, m, n, k, out_fmt=SLAB, out_bits=0)
    width = int(w[0].item())
    assert width == int(want.max().item()).bit_length()
    # the fused kernel (packed stages by TMA, 3-4 tiles per CTA), three runs: byte-identical to
    # the two-pass output, the int32 product included (a stage released too early showed up only
    # at this size, and not in every run)
    import ctypes as C

    from amethyst_b200 import _capi as A

    nb = m * ((n + 64 // width - 1) // (64 // width)) * 8
    try:
        A.check(A.lib().amx_set_tuning(C.byref(A.Tuning(0, 0, 2, 0))))
        for _ in range(3):
            f32, _ = ops.matmul(a, b, m, n, k, out_fmt=PLAIN32, out_bits=32)
            fs, fw = ops.matmul(a, b, m, n, k, out_fmt=SLAB, out_bits=0)
            torch.cuda.synchronize()
            assert torch.equal(f32.data[: 4 * m * n].view(torch.int32).long().reshape(m, n), got)
            assert int(fw[0].item()) == width and torch.equal(fs.data[:nb], o2.data[:nb])
    finally:
        A.check(A.lib().amx_set_tuning(None))


def test_batch_512_full_size(cuda):
    """512 columns, lengths log-uniform in [2^12, 2^24], widths 1..32, thresholds for
    selectivities uniform in [0.01, 0.99]: one batch run, every column checked."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    rng = np.random.default_rng(0xBA7C4)
    ncols = 512
    ns = np.exp(rng.uniform(np.log(2 ** 12), np.log(2 ** 24), ncols)).astype(np.int64)
    widths = rng.integers(1, 33, ncols)
    sel = rng.uniform(0.01, 0.99, ncols)
    cols, preds, vals, ts = [], [], [], []
    for i in range(ncols):
        cn, w = int(ns[i]), int(widths[i])
        v = values(cn, w, 0xC010 + i)
        t = max(1, int(round(sel[i] * (1 << w))))
        cols.append(ops.convert(plain_col(v, cn), SLAB, w))
        preds.append(ops.predicate(A.PRED_LT, t, 0, w))
        vals.append(v)
        ts.append(t)
    bt = ops.Batch(cols, preds)
    bt.run()
    bt.status()
    counts = bt.counts.cpu().numpy().view(np.uint64)
    sums = bt.sums.cpu().numpy().view(np.uint64)
    for i in range(ncols):
        v = vals[i].long() & 0xFFFFFFFF
        want = torch.masked_select(v, v < ts[i])
        assert int(counts[i]) == want.numel(), i
        assert int(sums[i]) == int(want.sum().item()) & 0xFFFFFFFFFFFFFFFF, i
        assert torch.equal(decoded(bt.outs[i], want.numel()), want), i
