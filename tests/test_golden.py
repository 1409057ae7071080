"""The C oracle against golden vectors produced by the reference's own host code
(tests/golden/make_golden.py).  Runs on any machine: the reference tree is not needed."""
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.mark.parametrize("name,fmt", [("slab", O.SLAB), ("nogaps", O.NOGAPS), ("plain64", O.PLAIN64)])
def test_accessors(g, name, fmt):
    words = g["words"]
    raw = np.concatenate([words, np.zeros(4, np.uint64)]).view(np.uint8)
    for b in range(1, 65):
        idx = g[f"{name}_{b}_idx"]
        n = int(idx.max()) + 1
        vals = O.decode(raw, n, fmt, b)
        assert np.array_equal(vals[idx.astype(np.int64)], g[f"{name}_{b}_val"]), (name, b)


def test_bitmask_accessor(g):
    words = g["words"]
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")
    assert np.array_equal(bits, g["bitmask_val"])
    # the oracle's mask convention (bit i%32 of uint32 word i/32) is the same bit order
    w32 = words.view(np.uint32)
    m = np.array([(w32[i // 32] >> (i % 32)) & 1 for i in range(0, 256 * 64, 7)], dtype=np.uint8)
    assert np.array_equal(m, g["bitmask_val"][::7])


def test_filter_predicate_half(g):
    for b in range(1, 65):
        got = [O.ora().ora_pred_eval(O.pred(9, bits=b), int(v) & ((1 << b) - 1)) for v in g["pred_in"]]
        assert np.array_equal(np.array(got, np.uint8), g["pred_half"][b - 1]), b


@pytest.mark.parametrize("op", [0, 2, 3, 4, 10, 11, 12])
def test_operators(g, op):
    l, r = g["op_l"], g["op_r"]
    want = g[f"op_{op}"]
    for ob in range(1, 65):
        got = [O.ora().ora_binop(op, int(a), int(c), ob) for a, c in zip(l, r)]
        assert np.array_equal(np.array(got, np.uint64), want[ob - 1]), (op, ob)


def test_out_width_rules(g):
    f = O.ora().ora_binop_out_bits
    assert [f(0, b, b) for b in range(1, 65)] == list(g["outbits_add"])
    assert [f(2, b, b) for b in range(1, 65)] == list(g["outbits_mul"])
    assert [f(4, b, b) for b in range(1, 65)] == list(g["outbits_mod"])


def test_reference_default_binary_op(g):
    """BINARY_OP as shipped is op_mul<2b> (src/config.cuh:74-85) while BINARY_OP_OUTBITS is
    b+1 (src/config.cuh:87-90): the oracle reproduces both halves of that mismatch."""
    l, r = g["op_l"], g["op_r"]
    for b in range(1, 65):
        m = (1 << b) - 1
        ob = min(2 * b, 64)
        got = [O.ora().ora_binop(2, int(a) & m, int(c) & m, ob) for a, c in zip(l, r)]
        assert np.array_equal(np.array(got, np.uint64), g["binary_op_default"][b - 1]), b
    assert list(g["binary_op_outbits"]) == [min(b + 1, 64) for b in range(1, 65)]


def test_pcg32(g):
    assert np.array_equal(O.pcg32(42, 1000), g["pcg32_seed42"])


def test_reference_inputs(g):
    d1, d2 = O.reference_inputs(42, 4096)
    assert np.array_equal(d1, g["main_data1"])
    assert np.array_equal(d2, g["main_data2"])


@pytest.mark.parametrize("sel", ["0.01", "0.1", "0.5", "0.9"])
def test_mask_generators(g, sel):
    n = 4096
    s = struct.unpack("f", struct.pack("f", float(sel)))[0]  # main() keeps selectivity in a float
    uni = O.mask_uniform(((n + 63) // 64) * 8, s)
    assert np.array_equal(uni[: n // 8], g[f"main_mask_0_{sel}"])
    assert np.array_equal(O.mask_clusters(s, 1, n), g[f"main_mask_1_{sel}"])
    assert np.array_equal(O.mask_clusters(s, 8, n), g[f"main_mask_2_{sel}"])
