"""The GPU data generators reproduce their host (numpy) definition exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits,eb", [(1, 4), (7, 4), (13, 4), (32, 4), (33, 8), (64, 8)])
def test_fill_uniform_matches_numpy(cuda, bits, eb):
    from amethyst_b200 import datagen

    n = 100003
    t = datagen.uniform_gpu(n, bits, 12345, eb)
    got = t[:n].cpu().numpy().view(np.uint32 if eb == 4 else np.uint64).astype(np.uint64)
    assert np.array_equal(got, datagen.uniform_np(12345, bits, n))


def test_fill_from_cdf_zipf(cuda):
    from amethyst_b200 import datagen

    n = 1 << 20
    cdf = datagen.zipf_cdf(1000, 1.1)
    t, _ = datagen.keys_from_cdf_gpu(n, cdf, 77)
    keys = t[:n].cpu().numpy()
    u = (datagen.draws_np(77, 0, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    want = np.searchsorted(cdf, u, side="right")
    assert np.array_equal(keys, want)
    assert keys.max() < 1000
