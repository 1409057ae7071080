"""Parity of the tile-pipeline operators (filter, compressstore, fused filter+compressstore,
binary ops, conversion, aggregation, chains) with the C oracle, bit-exact, through the C ABI.

Inputs carry random garbage in every unused bit (dead slab bits, bits above the width of
plain words, fields past n), as the reference's inputs do (src/main.cu:244-250).  Outputs are
compared as whole canonical buffers: dead bits and bits past the last element must be 0.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import FORMATS, NOGAPS, PLAIN32, PLAIN64, SLAB, gpu_bytes, make_column, to_gpu, valid_width

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 5, 31, 32, 33, 63, 64, 65, 1000, 4095, 4096, 4097, 8191, 9216, 15360, 40000, 100003]
WIDTHS = [1, 2, 3, 5, 7, 8, 11, 13, 14, 16, 17, 21, 31, 32, 33, 47, 63, 64]


def preds_for(bits):
    from amethyst_b200 import _capi as A

    top = (1 << bits) - 1
    half = 1 << (bits - 1)
    return [
        (A.PRED_LT, half // 5 + 1, 0),
        (A.PRED_GE, half, 0),
        (A.PRED_HALF, 0, 0),
        (A.PRED_BETWEEN, top // 4, top // 2),
        (A.PRED_EQ, top // 3, 0),
        (A.PRED_NE, 1, 0),
        (A.PRED_GT, top, 0),
        (A.PRED_ALL, 0, 0),
    ]


def cases(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        fmt = FORMATS[i % 4]
        bits = int(rng.choice([w for w in WIDTHS if valid_width(fmt, w)]))
        n = int(SIZES[i % len(SIZES)]) if i < 3 * len(SIZES) else int(rng.integers(1, 200000))
        out.append((fmt, bits, n, int(rng.integers(1, 1 << 30))))
    return out


@pytest.mark.parametrize("fmt,bits,n,seed", cases(1, 72))
def test_filter(cuda, fmt, bits, n, seed):
    from amethyst_b200 import ops

    v, raw = make_column(seed, fmt, bits, n)
    col = to_gpu(raw, n, fmt, bits)
    for kind, k0, k1 in preds_for(bits)[: 4 if n > 50000 else 8]:
        p = ops.predicate(kind, k0, k1, bits)
        got = ops.filter(col, p).cpu().numpy().view(np.uint32)[: (n + 31) // 32]
        want = O.filter(raw, n, fmt, bits, O.pred(kind, k0, k1, bits))
        assert np.array_equal(got, want), (fmt, bits, n, kind)


@pytest.mark.parametrize("fmt,bits,n,seed", cases(2, 72))
def test_filter_compressstore_same_format(cuda, fmt, bits, n, seed):
    from amethyst_b200 import ops

    v, raw = make_column(seed, fmt, bits, n)
    col = to_gpu(raw, n, fmt, bits)
    for kind, k0, k1 in preds_for(bits)[:4]:
        p = ops.predicate(kind, k0, k1, bits)
        out, cnt = ops.filter_compressstore(col, p, fmt, bits)
        want, wcnt = O.filter_compressstore(raw, n, fmt, bits, O.pred(kind, k0, k1, bits), fmt, bits)
        c = int(cnt[0].item())
        assert c == wcnt
        assert np.array_equal(gpu_bytes(out, c), want), (fmt, bits, n, kind)


@pytest.mark.parametrize("fmt,bits,n,seed", cases(3, 48))
def test_compressstore_any_output_format(cuda, fmt, bits, n, seed):
    from amethyst_b200 import ops

    v, raw = make_column(seed, fmt, bits, n)
    col = to_gpu(raw, n, fmt, bits)
    rng = np.random.default_rng(seed)
    words = (n + 31) // 32
    masks = [
        rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32),
        np.zeros(words, np.uint32),
        np.full(words, 0xFFFFFFFF, np.uint32),
        np.full(words, 0x55555555, np.uint32),
        (rng.random(words) < 0.02).astype(np.uint32) * np.uint32(0x80000001),
    ]
    import torch

    for mi, m in enumerate(masks):
        if n % 32 and words:
            m = m.copy()
            m[-1] &= np.uint32((1 << (n % 32)) - 1)
        dm = torch.zeros(words + 4, dtype=torch.int32, device="cuda")
        if words:
            dm[:words].copy_(torch.from_numpy(m.view(np.int32)))
        for ofmt in FORMATS:
            obits = bits if valid_width(ofmt, bits) else 32
            out, cnt = ops.compressstore(col, dm, ofmt, obits)
            want, wcnt = O.compressstore(raw, n, fmt, bits, m, ofmt, obits)
            c = int(cnt[0].item())
            assert c == wcnt, (mi, ofmt)
            assert np.array_equal(gpu_bytes(out, c), want), (fmt, bits, n, mi, ofmt, obits)


@pytest.mark.parametrize("fmt,bits,n,seed", cases(4, 48))
def test_convert_all_formats(cuda, fmt, bits, n, seed):
    from amethyst_b200 import ops

    v, raw = make_column(seed, fmt, bits, n)
    col = to_gpu(raw, n, fmt, bits)
    for ofmt in FORMATS:
        for obits in sorted({bits, max(1, bits - 3), min(64, bits + 5)}):
            if not valid_width(ofmt, obits):
                continue
            out = ops.convert(col, ofmt, obits)
            want = O.encode(ofmt, obits, v)[: O.storage_bytes(ofmt, obits, n)]
            assert np.array_equal(gpu_bytes(out), want), (fmt, bits, n, ofmt, obits)


@pytest.mark.parametrize("fmt,bits,n,seed", cases(5, 40))
def test_reduce(cuda, fmt, bits, n, seed):
    from amethyst_b200 import ops

    v, raw = make_column(seed, fmt, bits, n)
    col = to_gpu(raw, n, fmt, bits)
    for agg in range(6):
        got = int(ops.hop(agg, col).cpu().numpy().view(np.uint64)[0])
        assert got == O.reduce(agg, raw, n, fmt, bits), (fmt, bits, n, agg)


def binary_cases():
    from amethyst_b200 import _capi as A

    rng = np.random.default_rng(6)
    out = []
    ops = list(range(14))
    for i in range(70):
        op = ops[i % 14]
        lf, rf, of = (int(x) for x in rng.integers(0, 4, size=3))
        lb = int(rng.integers(1, 33 if lf == PLAIN32 else 65))
        rb = int(rng.integers(1, 33 if rf == PLAIN32 else 65))
        n = int([1, 7, 4096, 4097, 33333, 100000][i % 6])
        out.append((op, lf, lb, rf, rb, of, n, i + 11))
    # the reference's configurations and the chain config's widths
    for f in (SLAB, NOGAPS, PLAIN64):
        for b in (3, 11, 13, 31):
            out.append((A.OP_ADD, f, b, f, b, f, 50001, b))
            out.append((A.OP_MUL, f, b, f, b, f, 50001, b + 1))
    out.append((A.OP_ADD, SLAB, 7, SLAB, 13, SLAB, 123457, 5))
    out.append((A.OP_ADD, SLAB, 13, SLAB, 7, PLAIN32, 123457, 6))
    return out


@pytest.mark.parametrize("op,lf,lb,rf,rb,of,n,seed", binary_cases())
def test_binary(cuda, op, lf, lb, rf, rb, of, n, seed):
    from amethyst_b200 import ops
    from amethyst_b200._capi import lib

    lv, lraw = make_column(seed, lf, lb, n)
    rv, rraw = make_column(seed + 1, rf, rb, n)
    lc, rc = to_gpu(lraw, n, lf, lb), to_gpu(rraw, n, rf, rb)
    ob = int(lib().amx_binary_out_bits(op, lb, rb))
    if of == PLAIN32 and ob > 32:
        ob = 32
    for obits in sorted({ob, max(1, ob - 2)}):
        out = ops.binary_op(op, lc, rc, of, obits)
        want = O.binary(op, lraw, lf, lb, rraw, rf, rb, n, of, obits)
        assert np.array_equal(gpu_bytes(out), want), (op, lf, lb, rf, rb, of, obits, n)


def chain_cases():
    from amethyst_b200 import _capi as A

    out = []
    # configuration 2: A u7 + B u13 -> 14 bits, filter C >= 2^13 (and a ~50% variant), sum
    for lf, rf in [(SLAB, SLAB), (PLAIN32, PLAIN32), (SLAB, PLAIN32), (PLAIN32, SLAB)]:
        for of in (SLAB, PLAIN32, None):
            for k in (1 << 13, 4160):
                out.append((A.OP_ADD, lf, 7, rf, 13, 14, A.PRED_GE, k, of, 200003))
    out.append((A.OP_SUB, NOGAPS, 21, SLAB, 9, 21, A.PRED_LT, 5000, NOGAPS, 77777))
    out.append((A.OP_MUL, PLAIN64, 40, SLAB, 20, 60, A.PRED_BETWEEN, 1 << 40, PLAIN64, 50000))
    out.append((A.OP_ADD, SLAB, 11, SLAB, 11, 12, A.PRED_LT, 205, SLAB, 1 << 20))
    return out


@pytest.mark.parametrize("op,lf,lb,rf,rb,vb,pk,k0,of,n", chain_cases())
def test_chain(cuda, op, lf, lb, rf, rb, vb, pk, k0, of, n):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    lv, lraw = make_column(lb * 31 + n, lf, lb, n)
    rv, rraw = make_column(rb * 17 + n, rf, rb, n)
    lc, rc = to_gpu(lraw, n, lf, lb), to_gpu(rraw, n, rf, rb)
    k1 = (1 << 50) if pk == A.PRED_BETWEEN else 0
    p = ops.predicate(pk, k0, k1, vb)
    for agg in (A.AGG_SUM, A.AGG_MAX, A.AGG_MIN):
        out, mask, cnt, ag = ops.chain(lc, rc, op, vb, p, agg, out_fmt=of, out_bits=vb, want_mask=True)
        wout, wcnt, wagg = O.chain(op, (lraw, lf, lb), (rraw, rf, rb), vb, O.pred(pk, k0, k1, vb), agg, of, vb, n)
        c = int(cnt[0].item())
        assert c == wcnt
        assert int(ag.cpu().numpy().view(np.uint64)[0]) == wagg
        if of is not None:
            assert np.array_equal(gpu_bytes(out, c), wout)
        # the mask equals filtering the op result column
        vals = O.decode(O.binary(op, lraw, lf, lb, rraw, rf, rb, n, PLAIN64, vb), n, PLAIN64, vb)
        vraw = O.encode(PLAIN64, vb, vals)
        wmask = O.filter(vraw, n, PLAIN64, vb, O.pred(pk, k0, k1, vb))
        assert np.array_equal(mask.cpu().numpy().view(np.uint32)[: len(wmask)], wmask)


def test_chain_one_input_reduce_with_mask(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 300001
    v, raw = make_column(99, SLAB, 11, n)
    col = to_gpu(raw, n, SLAB, 11)
    m = np.random.default_rng(3).integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    m[-1] &= np.uint32((1 << (n % 32)) - 1)
    dm = torch.zeros(len(m) + 4, dtype=torch.int32, device="cuda")
    dm[: len(m)].copy_(torch.from_numpy(m.view(np.int32)))
    for agg in range(6):
        got = int(ops.hop(agg, col, dm).cpu().numpy().view(np.uint64)[0])
        assert got == O.reduce(agg, raw, n, SLAB, 11, m)


def test_policies_agree(cuda):
    """The compile-time-width policy and the generic runtime-width policy give equal bytes."""
    import ctypes as C

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 250007
    for bits in (1, 2, 3, 7, 11, 13, 16, 21, 32):
        v, raw = make_column(bits, SLAB, bits, n)
        col = to_gpu(raw, n, SLAB, bits)
        p = ops.predicate(A.PRED_LT, (1 << bits) // 3 + 1, 0, bits)
        out, cnt = ops.filter_compressstore(col, p, SLAB, bits)
        want, wcnt = O.filter_compressstore(raw, n, SLAB, bits, O.pred(A.PRED_LT, (1 << bits) // 3 + 1, 0, bits),
                                            SLAB, bits)
        assert int(cnt[0].item()) == wcnt
        assert np.array_equal(gpu_bytes(out, wcnt), want)


def test_repeated_calls_reuse_workspace(cuda):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 1 << 20
    v, raw = make_column(5, SLAB, 11, n)
    col = to_gpu(raw, n, SLAB, 11)
    ws = ops.workspace(n)
    p = ops.predicate(A.PRED_LT, 205, 0, 11)
    want, wcnt = O.filter_compressstore(raw, n, SLAB, 11, O.pred(A.PRED_LT, 205), SLAB, 11)
    for _ in range(3):
        out, cnt = ops.filter_compressstore(col, p, SLAB, 11, ws=ws)
        assert int(cnt[0].item()) == wcnt
        assert np.array_equal(gpu_bytes(out, wcnt), want)
    ops.workspace_status(ws)


def plain_pair_cases():
    from amethyst_b200 import _capi as A

    ops8 = [A.OP_ADD, A.OP_SUB, A.OP_MUL, A.OP_MIN, A.OP_MAX, A.OP_AND, A.OP_OR, A.OP_XOR]
    out = []
    for lb, rb in [(7, 13), (13, 7), (11, 11), (13, 13)]:
        for op in ops8:
            out.append((op, lb, rb))
    return out


@pytest.mark.parametrize("op,lb,rb", plain_pair_cases())
def test_chain_plain_pair_kernels(cuda, op, lb, rb):
    """Compacting chains with no mask out and a sum or nothing (the plain two-column kernels, one
    per slab-width pair and op) and with another aggregate (the general kernel), into slabs of
    the op's natural width (compile-time encoder), other slab widths, plain32 and nogaps."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    vb = int(A.lib().amx_binary_out_bits(op, lb, rb))
    for n in (200003, 1 << 20):
        lv, lraw = make_column(lb * 13 + op + n, SLAB, lb, n)
        rv, rraw = make_column(rb * 29 + op + n, SLAB, rb, n)
        lc, rc = to_gpu(lraw, n, SLAB, lb), to_gpu(rraw, n, SLAB, rb)
        top = (1 << vb) - 1
        for pk, k0 in [(A.PRED_LT, top // 3 + 1), (A.PRED_GE, top // 2)]:
            p = ops.predicate(pk, k0, 0, vb)
            for agg, want_agg in [(A.AGG_SUM, True), (A.AGG_SUM, False), (A.AGG_MAX, True)]:
                for of, ob in [(SLAB, vb), (SLAB, 16), (PLAIN32, 32), (NOGAPS, vb)]:
                    out, _, cnt, ag = ops.chain(lc, rc, op, vb, p, agg, out_fmt=of, out_bits=ob, want_agg=want_agg)
                    wout, wcnt, wagg = O.chain(op, (lraw, SLAB, lb), (rraw, SLAB, rb), vb, O.pred(pk, k0, 0, vb), agg,
                                               of, ob, n)
                    c = int(cnt[0].item())
                    assert c == wcnt, (op, lb, rb, n, pk, agg, of, ob)
                    if want_agg:
                        assert int(ag.cpu().numpy().view(np.uint64)[0]) == wagg, (op, lb, rb, n, pk, agg)
                    assert np.array_equal(gpu_bytes(out, c), wout), (op, lb, rb, n, pk, agg, of, ob)


@pytest.mark.parametrize("lf,lb,rf,rb,op", [
    (PLAIN32, 7, PLAIN32, 13, 0), (PLAIN32, 12, NOGAPS, 9, 1), (NOGAPS, 5, PLAIN64, 11, 9),
    (PLAIN64, 14, SLAB, 14, 6), (SLAB, 6, SLAB, 9, 2), (PLAIN32, 16, PLAIN32, 16, 5)])
def test_chain_plain_generic_kernel(cuda, lf, lb, rf, rb, op):
    """Compacting chains outside the compile-time width pairs, with no mask out and a sum or
    nothing (the plain variant of the runtime-format policy) or another aggregate (the general
    one), against the oracle."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    vb = int(A.lib().amx_binary_out_bits(op, lb, rb))
    for n in (1, 6143, 6145, 300007):
        lv, lraw = make_column(lb * 7 + op + n, lf, lb, n)
        rv, rraw = make_column(rb * 5 + op + n, rf, rb, n)
        lc, rc = to_gpu(lraw, n, lf, lb), to_gpu(rraw, n, rf, rb)
        top = (1 << vb) - 1
        p = ops.predicate(A.PRED_BETWEEN, top // 5, top // 2, vb)
        for agg, want_agg in [(A.AGG_SUM, True), (A.AGG_SUM, False), (A.AGG_XOR, True)]:
            for of, ob in [(SLAB, vb), (PLAIN32, 32), (NOGAPS, vb)]:
                out, _, cnt, ag = ops.chain(lc, rc, op, vb, p, agg, out_fmt=of, out_bits=ob, want_agg=want_agg)
                wout, wcnt, wagg = O.chain(op, (lraw, lf, lb), (rraw, rf, rb), vb,
                                           O.pred(A.PRED_BETWEEN, top // 5, top // 2, vb), agg, of, ob, n)
                c = int(cnt[0].item())
                assert c == wcnt, (lf, lb, rf, rb, op, n, agg, of)
                if want_agg:
                    assert int(ag.cpu().numpy().view(np.uint64)[0]) == wagg, (lf, lb, rf, rb, op, n, agg)
                assert np.array_equal(gpu_bytes(out, c), wout), (lf, lb, rf, rb, op, n, agg, of)


# The runtime-format map variant (12 elements per thread) serves element-wise outputs only where
# its stage pair and output slot fit in 220 KB: 5632 + slot + 2 * stage <= 225280 bytes, with
# slot = 6144 * (2 or 8) bytes and stage = the staged bytes of both inputs for 6144 elements.
# These cases sit on both sides of that line (the other side runs the 8-element kernel), with
# ragged lengths, so both kernels are pinned to the oracle.
MAP_FIT_CASES = [
    # op, lhs (fmt, bits), rhs (fmt, bits) or None, out (fmt, bits), fits
    (None, (PLAIN64, 64), None, (PLAIN64, 64), True),                   # convert: 153,344 B
    (0, (PLAIN64, 64), (PLAIN32, 32), (PLAIN64, 64), True),             # 202,752 B
    (0, (PLAIN64, 64), (NOGAPS, 40), (NOGAPS, 64), True),               # 215,040 B
    (9, (PLAIN64, 64), (NOGAPS, 48), (PLAIN64, 64), False),             # 227,328 B
    (0, (PLAIN64, 64), (PLAIN64, 63), (SLAB, 64), False),               # 251,904 B
    (2, (SLAB, 33), (PLAIN64, 30), (NOGAPS, 63), False),                # 251,904 B
    (1, (NOGAPS, 60), (PLAIN32, 16), (PLAIN32, 16), True),              # 16-bit slot
]


@pytest.mark.parametrize("case", range(len(MAP_FIT_CASES)))
@pytest.mark.parametrize("n", [6144 * 3 + 1, 6144 * 5 - 1, 100003])
def test_map_variant_fit_boundary(cuda, case, n):
    from amethyst_b200 import ops

    op, (lf, lb), rhs, (of, ob), _ = MAP_FIT_CASES[case]
    lv, lraw = make_column(case * 101 + n, lf, lb, n)
    lc = to_gpu(lraw, n, lf, lb)
    if rhs is None:
        out = ops.convert(lc, of, ob)
        want = O.binary(13, lraw, lf, lb, lraw, lf, lb, n, of, ob)  # LHS = identity
    else:
        rf, rb = rhs
        rv, rraw = make_column(case * 103 + n, rf, rb, n)
        out = ops.binary_op(op, lc, to_gpu(rraw, n, rf, rb), of, ob)
        want = O.binary(op, lraw, lf, lb, rraw, rf, rb, n, of, ob)
    assert np.array_equal(gpu_bytes(out), want), (MAP_FIT_CASES[case], n)


def test_map_fit_table_matches_the_rule():
    """The byte counts behind MAP_FIT_CASES, recomputed from the staging rule."""
    def stage(fmt, bits, t=6144):
        b = {PLAIN32: 4 * t, PLAIN64: 8 * t, SLAB: 8 * (t // (64 // bits) + 2),
             NOGAPS: 8 * (t * bits // 64 + 2)}[fmt]
        return (b + 48 + 127) // 128 * 128

    for op, (lf, lb), rhs, (of, ob), fits in MAP_FIT_CASES:
        vbits = ob
        st = stage(lf, lb) + (stage(*rhs) if rhs else 0)
        slot = (6144 * (2 if vbits <= 16 else 8) + 127) // 128 * 128
        assert (5632 + slot + 2 * st <= 225280) == fits, (lf, lb, rhs, of, ob)
