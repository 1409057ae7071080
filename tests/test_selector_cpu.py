"""Host logic of the format selector: the synthetic chain distribution, the features and the
storage-width rule (no GPU needed)."""
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


def test_features_are_bounded_and_deterministic():
    rng = np.random.default_rng(1)
    for k in range(200):
        c = S.random_chain(rng, seed=k)
        for i, op in enumerate(c.ops):
            f = S.features(c, i, c.n, c.bits, S.natural_out_bits(op.kind, c.bits, op.rhs_bits))
            assert f.shape == (16,) and f.dtype == np.float32
            assert np.all(f >= 0) and np.all(f <= 1.0 + 1e-6)
            assert np.array_equal(f, S.features(c, i, c.n, c.bits, S.natural_out_bits(op.kind, c.bits, op.rhs_bits)))


def test_storage_widths():
    assert S.candidate_bits(2, 5) == 8 and S.candidate_bits(2, 9) == 16 and S.candidate_bits(2, 17) == 32
    assert S.candidate_bits(2, 5, "sub") == 5  # subtraction wraps at its natural width
    assert S.candidate_bits(1, 13) == 13
    assert S.natural_out_bits("add", 31, 5) == 32 and S.natural_out_bits("mul", 20, 16) == 32
