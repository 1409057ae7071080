"""Host logic of the format selector: the synthetic chain distribution, the features, the
candidates of a decision point and the value bounds behind the tightest width (no GPU needed)."""
import numpy as np

from amethyst_b200 import chains as S


def test_random_chains_follow_the_stated_distribution():
    rng = np.random.default_rng(0)
    chains = [S.random_chain(rng, seed=i) for i in range(2000)]
    lengths = [len(c.ops) for c in chains]
    assert min(lengths) == 2 and max(lengths) == 5
    assert min(c.bits for c in chains) == 1 and max(c.bits for c in chains) == 32
    assert all(2 ** 16 <= c.n <= 2 ** 26 for c in chains)
    kinds = {o.kind for c in chains for o in c.ops}
    assert kinds == set(S.OPS)
    sels = [o.sel for c in chains for o in c.ops]
    assert 0.01 <= min(sels) and max(sels) <= 0.99
    groups = [o.groups for c in chains for o in c.ops]
    assert 2 <= min(groups) and max(groups) <= 2 ** 16


def test_features_are_bounded_and_choice_independent():
    rng = np.random.default_rng(1)
    hist = np.bincount(np.arange(1, 1000) % 20, minlength=65)
    for k in range(300):
        c = S.random_chain(rng, seed=k)
        runs = []
        for choose in (S.fixed(0), S.fixed(4), S.fixed(5)):
            feats = []
            S.plan(c, lambda i, f, valid: (feats.append(f), choose(i, f, valid))[1], hist)
            runs.append(np.array(feats, np.float32).reshape(-1, 16))
        for f in runs:
            assert f.shape == (len(S.decision_points(c)), 16) and f.dtype == np.float32
            assert np.all(f >= 0) and np.all(f <= 1.0 + 1e-6)
        assert all(np.array_equal(runs[0], f) for f in runs[1:])


def test_candidates():
    assert S.candidate_storage(2, 5, 31) == (S.SLAB, 8)
    assert S.candidate_storage(2, 9, 511) == (S.SLAB, 16) and S.candidate_storage(2, 17, 1) == (S.SLAB, 32)
    assert S.candidate_storage(1, 13, 5) == (S.SLAB, 13)
    assert S.candidate_storage(4, 13, 5) == (S.SLAB, 3) and S.candidate_storage(4, 13, 0) == (S.SLAB, 1)
    assert S.candidate_storage(0, 13, 5) == (S.PLAIN32, 13) and S.candidate_storage(3, 13, 5) == (S.NOGAPS, 13)
    assert S.natural_out_bits("add", 31, 5) == 32 and S.natural_out_bits("mul", 20, 16) == 32
    ch = S.ChainSpec(100, 8, [S.OpSpec("add", rhs_bits=3), S.OpSpec("compressstore", sel=0.5), S.OpSpec("mul", rhs_bits=2),
                              S.OpSpec("sum")])
    assert S.candidate_valid(ch, 0, S.FUSED) and not S.candidate_valid(ch, 2, S.FUSED)
    assert not S.candidate_valid(ch, 1, S.FUSED)
    assert len(S.valid_combos(ch)) == 6 * 5 * 5
    ch2 = S.ChainSpec(100, 8, [S.OpSpec("sub", rhs_bits=3), S.OpSpec("filter", sel=0.5), S.OpSpec("compressstore")])
    assert S.candidate_valid(ch2, 0, S.FUSED)
    ch2.ops[2] = S.OpSpec("sum")
    assert not S.candidate_valid(ch2, 0, S.FUSED)


def _simulate(chain):
    """The chain's values in numpy; returns, per decision point, the largest value produced."""
    from amethyst_b200 import datagen

    x = datagen.uniform_np(chain.seed + 1, chain.bits, chain.n)
    steps, _ = S.plan(chain, S.fixed(S.DEFAULT_CHOICE))
    mask = None
    peaks = []
    for i, st in enumerate(steps):
        if st[0] == "filter":
            mask = x < np.uint64(st[1])
        elif st[0] == "compressstore":
            x = x[mask] if mask is not None else x[x < np.uint64(st[1])]
            mask = None
            peaks.append(int(x.max()) if x.size else 0)
        elif st[0] == "binary":
            y = datagen.uniform_np(chain.seed + 17 + i, chain.ops[i].rhs_bits, chain.n)[: x.size]
            m = np.uint64((1 << st[2]) - 1)
            with np.errstate(over="ignore"):
                v = {0: x + y, 1: x - y, 2: x * y}[st[1]]
            x = v & m
            peaks.append(int(x.max()) if x.size else 0)
    return peaks


def test_tight_width_holds_every_value():
    """The value bound the planner tracks (through filters, compressstores and ops that may
    wrap) never underestimates: slabs at the tightest width lose no value."""
    rng = np.random.default_rng(5)
    for k in range(400):
        ch = S.random_chain(rng, seed=k, n_range=(8, 12))
        peaks = _simulate(ch)
        steps, _ = S.plan(ch, S.fixed(4))
        tight = [st[3] if st[0] == "compressstore" else st[4] for st in steps if st[0] in ("compressstore", "binary")]
        assert len(tight) == len(peaks)
        for w, p in zip(tight, peaks):
            assert p < (1 << w), ([o.kind for o in ch.ops], w, p)
