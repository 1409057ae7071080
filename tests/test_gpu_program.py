"""Operator-chain programs (amx_program_*) and their CUDA graphs, against the C oracle.

Every chain runs (a) as a program under every combination of candidates -- storage formats,
widths and the fused kernel variant -- with lengths kept on the device, (b) in the plain
per-operator form through the single-operator C ABI, and (c) on the C oracle operator by
operator (tests/chain_ref.py).  All digests (aggregates, survivor counts, group tables and the
final column's values) must be identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chains(seed, count, n_range, max_dp=3):
    from amethyst_b200 import chains as X

    rng = np.random.default_rng(seed)
    out = []
    k = 0
    while len(out) < count:
        ch = X.random_chain(rng, seed=seed * 1000 + k, n_range=n_range)
        k += 1
        if len(X.decision_points(ch)) <= max_dp:
            out.append(ch)
    return out


def test_every_candidate_combination_matches_the_oracle(cuda):
    import chain_ref

    from amethyst_b200 import chains as X
    from amethyst_b200 import selector as S

    checked = 0
    for ch in _chains(3, 24, (10, 17)):
        r = S.ChainRunner(ch)
        want = chain_ref.run(r)
        r.clear_results()
        xd = r.run_plain()
        assert r.digest(r.plain_final_column(xd)) == want, ([o.kind for o in ch.ops], "plain")
        for combo in X.valid_combos(ch):
            got = r.program_digest(X.from_combo(combo))
            assert got == want, ([o.kind for o in ch.ops], ch.n, ch.bits, combo)
            checked += 1
    assert checked > 100


def test_edge_chains(cuda):
    """Empty survivors followed by more operators, a filter then a binary op then a
    compressstore (the mask outlives the op), ragged lengths around tile sizes, n = 1, and the
    step pairs a program runs as one pass (filter + compressstore, a reduce inside the pass
    before it, a fused op ahead of a filter + compressstore)."""
    import chain_ref

    from amethyst_b200 import chains as X
    from amethyst_b200 import selector as S

    O = X.OpSpec
    cases = [
        X.ChainSpec(5000, 20, [O("compressstore", sel=0.000001), O("add", rhs_bits=7), O("sum"), O("groupby", groups=40)], 1),
        X.ChainSpec(70001, 12, [O("filter", sel=0.3), O("mul", rhs_bits=5), O("compressstore"), O("max")], 2),
        X.ChainSpec(4097, 32, [O("sub", rhs_bits=16), O("compressstore", sel=0.5), O("min"), O("add", rhs_bits=3)], 3),
        X.ChainSpec(1, 1, [O("add", rhs_bits=1), O("compressstore", sel=0.99), O("sum")], 4),
        X.ChainSpec(6144 * 3 + 5, 20, [O("filter", sel=0.6), O("groupby", groups=5000), O("compressstore"),
                                         O("groupby", groups=3)], 5),
        X.ChainSpec(200000, 3, [O("mul", rhs_bits=16), O("compressstore", sel=0.02), O("mul", rhs_bits=16),
                                O("compressstore", sel=0.7), O("sum")], 6),
        # steps the program merges into one pass
        X.ChainSpec(300001, 14, [O("filter", sel=0.3), O("compressstore"), O("sum"), O("max")], 7),
        X.ChainSpec(300001, 9, [O("add", rhs_bits=12), O("filter", sel=0.5), O("compressstore"), O("min")], 8),
        X.ChainSpec(123457, 21, [O("filter", sel=0.7), O("max"), O("mul", rhs_bits=3), O("sum")], 9),
        X.ChainSpec(123457, 5, [O("sub", rhs_bits=9), O("sum"), O("filter", sel=0.1), O("add", rhs_bits=2),
                                O("sum")], 10),
    ]
    for ch in cases:
        r = S.ChainRunner(ch)
        want = chain_ref.run(r)
        for combo in X.valid_combos(ch):
            assert r.program_digest(X.from_combo(combo)) == want, ([o.kind for o in ch.ops], combo)
        r.clear_results()
        xd = r.run_plain()
        assert r.digest(r.plain_final_column(xd)) == want


def test_graph_of_many_programs_matches_single_runs(cuda):
    """Programs of many chains captured into one graph over four lanes, replayed twice: each
    chain's digest equals its oracle digest."""
    import torch

    import chain_ref

    from amethyst_b200 import chains as X
    from amethyst_b200 import ops
    from amethyst_b200 import selector as S

    chains = _chains(9, 20, (12, 19), max_dp=5)
    results = torch.zeros(sum(len(c.ops) for c in chains), dtype=torch.int64, device="cuda")
    runners, progs, slot = [], [], 0
    rng = np.random.default_rng(4)
    for ch in chains:
        r = S.ChainRunner(ch, results, slot)
        slot += len(ch.ops)
        combos = X.valid_combos(ch)
        prog, _ = r.program(X.from_combo(combos[int(rng.integers(0, len(combos)))]))
        runners.append(r)
        progs.append(prog)
    wants = [chain_ref.run(r) for r in runners]
    g = ops.Graph(progs, lanes=4)
    for _ in range(2):
        results.zero_()
        g.launch()
        torch.cuda.synchronize()
        for r, p, w in zip(runners, progs, wants):
            assert r.digest(r.final_column(p)) == w
    for p in progs:
        p.status()


def test_program_validation(cuda):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    x = ops.PackedColumn.empty(1000, A.SLAB, 11)
    aux = ops.PackedColumn.empty(1000, A.SLAB, 5)
    short = ops.PackedColumn.empty(999, A.SLAB, 5)
    fused = A.Step(kind=A.STEP_BINARY, op=A.OP_ADD, value_bits=12, out_format=A.FORMAT_FUSED, out_bits=12,
                   aux=aux.desc)
    red = A.Step(kind=A.STEP_REDUCE, op=A.AGG_SUM, d_result=x.data.data_ptr())
    with pytest.raises(A.AmxError) as e:
        ops.Program(x, [fused, red])  # a fused op must precede a compressstore
    assert e.value.status == 1
    bad = A.Step(kind=A.STEP_BINARY, op=A.OP_ADD, value_bits=12, out_format=A.SLAB, out_bits=12, aux=short.desc)
    with pytest.raises(A.AmxError):
        ops.Program(x, [bad])
    with pytest.raises(A.AmxError) as e:
        ops.Program(x, [red] * 33)
    assert e.value.status == 7
    nores = A.Step(kind=A.STEP_REDUCE, op=A.AGG_SUM)
    with pytest.raises(A.AmxError):
        ops.Program(x, [nores])


def test_bit_histogram_matches_numpy(cuda):
    from amethyst_b200 import ops
    from helpers import FORMATS, make_column, to_gpu, valid_width

    for fmt in FORMATS:
        for bits in (1, 7, 13, 32, 33, 64):
            if not valid_width(fmt, bits):
                continue
            for n in (1, 31, 1000, 100003):
                v, raw = make_column(bits * 7 + n, fmt, bits, n)
                h = ops.bit_histogram(to_gpu(raw, n, fmt, bits)).cpu().numpy()
                lens = np.array([int(x).bit_length() for x in v])
                assert np.array_equal(h, np.bincount(lens, minlength=65)), (fmt, bits, n)
