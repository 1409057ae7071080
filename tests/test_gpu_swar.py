"""The field-parallel slab policy (whole-word predicate evaluation) against the C oracle,
bit-exact, for every slab width 1..32 and for predicates at the edges of the value range
(empty, full, wrap-around and complemented intervals).  Each case runs with the policy forced
and with the automatic choice, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import SLAB, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu

SWAR_BASE = 200


def edge_preds(bits):
    from amethyst_b200 import _capi as A

    top = (1 << bits) - 1
    half = 1 << (bits - 1)
    return [
        (A.PRED_LT, max(1, top // 10), 0),
        (A.PRED_LT, 0, 0),                  # nothing passes
        (A.PRED_LE, top, 0),                # everything passes
        (A.PRED_GE, half, 0),               # lower bound on the field's top bit
        (A.PRED_GE, half - 1 if half > 1 else 1, 0),
        (A.PRED_GT, top, 0),                # nothing passes
        (A.PRED_GT, top - 1, 0),            # only the maximum
        (A.PRED_EQ, 0, 0),
        (A.PRED_EQ, top, 0),
        (A.PRED_NE, top // 3, 0),           # complement of a point
        (A.PRED_BETWEEN, top // 4, top - top // 4),
        (A.PRED_BETWEEN, top, top // 2),    # k0 > k1: empty range
        (A.PRED_NOT_BETWEEN, top // 3, top // 2),
        (A.PRED_NOT_BETWEEN, 0, top),       # nothing passes
        (A.PRED_HALF, 0, 0),
        (A.PRED_ALL, 0, 0),
        (A.PRED_GE, top + 5, 0),            # bound beyond the width: nothing passes
        (A.PRED_LT, top + 5, 0),            # bound beyond the width: everything passes
    ]


def _set_policy(pid):
    from amethyst_b200 import _capi as A

    t = A.Tuning(0, 0, pid, 0)
    A.check(A.lib().amx_set_tuning(C.byref(t)))


@pytest.fixture
def restore_tuning():
    yield
    from amethyst_b200 import _capi as A

    A.check(A.lib().amx_set_tuning(None))


@pytest.mark.parametrize("bits", list(range(1, 33)))
def test_swar_filter_and_compressstore(cuda, restore_tuning, bits):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = [100003, 77777, 40961, 1 << 17][bits % 4]
    v, raw = make_column(bits * 31 + 7, SLAB, bits, n)
    col = to_gpu(raw, n, SLAB, bits)
    for force in (1 + SWAR_BASE + bits, 0):
        _set_policy(force)
        for kind, k0, k1 in edge_preds(bits):
            p = ops.predicate(kind, k0, k1, bits)
            op = O.pred(kind, k0, k1, bits)
            got = ops.filter(col, p).cpu().numpy().view(np.uint32)[: (n + 31) // 32]
            assert np.array_equal(got, O.filter(raw, n, SLAB, bits, op)), ("filter", bits, kind, k0, k1)
            out, cnt = ops.filter_compressstore(col, p, SLAB, bits)
            want, wcnt = O.filter_compressstore(raw, n, SLAB, bits, op, SLAB, bits)
            assert int(cnt[0].item()) == wcnt, ("count", bits, kind, k0, k1)
            assert np.array_equal(gpu_bytes(out, wcnt), want), ("compressstore", bits, kind, k0, k1)


@pytest.mark.parametrize("bits", [1, 3, 7, 8, 11, 13, 16, 21, 32])
@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 4097, 32767, 32768, 32769, 262145])
def test_swar_chain_outputs(cuda, restore_tuning, bits, n):
    """Count, every aggregation, the mask and the compacted column in plain32 and nogaps, one
    slab column with a predicate (policy forced), at sizes around tile edges."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    v, raw = make_column(bits * 7 + n, SLAB, bits, n)
    col = to_gpu(raw, n, SLAB, bits)
    _set_policy(1 + SWAR_BASE + bits)
    top = (1 << bits) - 1
    for kind, k0, k1 in [(A.PRED_LT, top // 3 + 1, 0), (A.PRED_NOT_BETWEEN, top // 5, top // 2)]:
        p = ops.predicate(kind, k0, k1, bits)
        op = O.pred(kind, k0, k1, bits)
        for agg in range(6):
            for out_fmt, out_bits in [(A.PLAIN32, 32), (A.NOGAPS, bits), (None, None)]:
                out, mask, cnt, ag = ops.chain(col, None, A.OP_LHS, bits, p, agg, out_fmt=out_fmt,
                                               out_bits=out_bits, want_mask=True)
                wout, wcnt, wagg = O.chain(A.OP_LHS, (raw, SLAB, bits), None, bits, op, agg, out_fmt, out_bits, n)
                assert int(cnt[0].item()) == wcnt
                assert int(ag.cpu().numpy().view(np.uint64)[0]) == wagg, (bits, n, kind, agg)
                gm = mask.cpu().numpy().view(np.uint32)[: (n + 31) // 32]
                assert np.array_equal(gm, O.filter(raw, n, SLAB, bits, op))
                if out_fmt is not None:
                    assert np.array_equal(gpu_bytes(out, wcnt), wout), (bits, n, kind, out_fmt)


@pytest.mark.parametrize("bits", [1, 5, 8, 11, 13, 16, 24, 32])
@pytest.mark.parametrize("n", [0, 1, 4097, 32769, 300001])
def test_swar_count_and_aggregate_only(cuda, restore_tuning, bits, n):
    """Count and every aggregation with no output column and no bitmask (the count-and-aggregate
    variant of the field-parallel kernel), automatic policy choice."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    v, raw = make_column(bits * 11 + n, SLAB, bits, n)
    col = to_gpu(raw, n, SLAB, bits)
    top = (1 << bits) - 1
    for kind, k0, k1 in [(A.PRED_LT, top // 3 + 1, 0), (A.PRED_BETWEEN, top // 5, top // 2), (A.PRED_ALL, 0, 0)]:
        p = ops.predicate(kind, k0, k1, bits)
        op = O.pred(kind, k0, k1, bits)
        for agg in range(6):
            _, _, cnt, ag = ops.chain(col, None, A.OP_LHS, bits, p, agg)
            _, wcnt, wagg = O.chain(A.OP_LHS, (raw, SLAB, bits), None, bits, op, agg, None, None, n)
            assert int(cnt[0].item()) == wcnt, (bits, n, kind, agg)
            assert int(ag.cpu().numpy().view(np.uint64)[0]) == wagg, (bits, n, kind, agg)


def _masks(n, seed):
    """Input masks of n elements (LSB-first uint32 words, bits past n clear): random, none, all,
    alternating, sparse, and runs that start and end inside words."""
    rng = np.random.default_rng(seed)
    words = (n + 31) // 32
    runs = np.zeros(n, bool)
    for a in rng.integers(0, max(n, 1), size=12):
        runs[a : a + int(rng.integers(1, 5000))] = True
    out = [
        rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32),
        np.zeros(words, np.uint32),
        np.full(words, 0xFFFFFFFF, np.uint32),
        np.full(words, 0xAAAAAAAA, np.uint32),
        (rng.random(words) < 0.03).astype(np.uint32) * np.uint32(0x00010001),
        np.packbits(np.concatenate([runs, np.zeros(words * 32 - n, bool)]), bitorder="little").view(np.uint32)
        if words else np.zeros(0, np.uint32),
    ]
    for m in out:
        if n % 32 and words:
            m[-1] &= np.uint32((1 << (n % 32)) - 1)
    return out


@pytest.mark.parametrize("bits", list(range(1, 33)))
def test_swar_mask_input(cuda, restore_tuning, bits):
    """compressstore by a given mask (slabs at the input width: the plain variant up to 16 bits;
    plain32 and nogaps: the general variant) and masked aggregates (the count-and-aggregate
    variant), field-parallel policy forced and automatic, against the oracle bit-exact."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = [100003, 77777, 40961, (1 << 17) + 5][bits % 4]
    v, raw = make_column(bits * 13 + 3, SLAB, bits, n)
    col = to_gpu(raw, n, SLAB, bits)
    words = (n + 31) // 32
    for force in (1 + SWAR_BASE + bits, 0):
        _set_policy(force)
        for mi, m in enumerate(_masks(n, bits)):
            dm = torch.zeros(words + 4, dtype=torch.int32, device="cuda")
            dm[:words].copy_(torch.from_numpy(m.view(np.int32)))
            for ofmt, obits in [(SLAB, bits), (A.PLAIN32, 32), (A.NOGAPS, bits)]:
                out, cnt = ops.compressstore(col, dm, ofmt, obits)
                want, wcnt = O.compressstore(raw, n, SLAB, bits, m, ofmt, obits)
                assert int(cnt[0].item()) == wcnt, (bits, mi, ofmt)
                assert np.array_equal(gpu_bytes(out, wcnt), want), (bits, mi, ofmt)
            for agg in (A.AGG_SUM, A.AGG_MAX, A.AGG_XOR):
                got = int(ops.reduce(agg, col, dm).cpu().numpy().view(np.uint64)[0])
                assert got == O.reduce(agg, raw, n, SLAB, bits, m), (bits, mi, agg)


@pytest.mark.parametrize("bits", list(range(1, 33)))
def test_sum_alone_every_width(cuda, restore_tuning, bits):
    """A sum with neither predicate nor mask (field-parallel lanes, bit planes at 1-3 bits, a field
    visit or the compile-time policy, by width): random columns and columns of maximal fields,
    ragged tails, against the oracle bit-exact; forced and automatic policy choice agree."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    top = (1 << bits) - 1
    for n in (1, 4097, 300001):
        _, raw = make_column(bits * 17 + n, SLAB, bits, n)
        full = O.encode(SLAB, bits, np.full(n, top, np.uint64))
        for r in (raw, full):
            col = to_gpu(r, n, SLAB, bits)
            want = O.reduce(A.AGG_SUM, r, n, SLAB, bits)
            for force in (0, 1 + SWAR_BASE + bits):
                _set_policy(force)
                got = int(ops.hop(A.AGG_SUM, col).cpu().numpy().view(np.uint64)[0])
                assert got == want, (bits, n, force)
