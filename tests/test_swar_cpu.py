"""The multiplication tricks of the field-parallel slab policy (amethyst_b200/csrc/amx_swar.cuh),
checked on the host.  The flag gather (swar_gather_flags): for every width B = 8..32 and every
pattern of the floor(64/B) field flags, (g * M) >> (E(B-1)) & (2^E - 1) equals the pattern; at
B = 7 it does not, so the kernel keeps the per-field loop below B = 8.  The flag deposit
(swar_deposit_flags), which puts an input mask's bits on the field tops: for every width 1..32
against bit-by-bit placement, exhaustively up to 2^21 patterns and on random patterns above."""
import numpy as np

M64 = (1 << 64) - 1


def gather_mul(b):
    e = 64 // b
    return sum(1 << ((e - 1 - j) * (b - 1)) for j in range(e))


def test_flag_gather_is_exact_for_every_pattern():
    for b in range(8, 33):
        e = 64 // b
        m = gather_mul(b)
        for pattern in range(1 << e):
            g = 0
            for k in range(e):
                if (pattern >> k) & 1:
                    g |= 1 << (k * b + b - 1)  # the top bit of field k
            got = (((g * m) & ((1 << 64) - 1)) >> (e * (b - 1))) & ((1 << e) - 1)
            assert got == pattern, (b, pattern)


def test_the_gather_fails_below_eight_bits():
    b, e = 7, 9
    m = sum(1 << ((e - 1 - j) * (b - 1)) for j in range(e))
    bad = 0
    for pattern in range(1 << e):
        g = sum(1 << (k * b + b - 1) for k in range(e) if (pattern >> k) & 1)
        got = (((g * m) & ((1 << 64) - 1)) >> (e * (b - 1))) & ((1 << e) - 1)
        bad += got != pattern
    assert bad > 0


def top_bits(b):
    return sum(1 << (k * b + b - 1) for k in range(64 // b))


def deposit(b, m):
    """swar_deposit_flags<b>(m) on numpy uint64 arrays (products wrap modulo 2^64 as on the GPU)."""
    m = m.astype(np.uint64)
    if b == 1:
        return m
    e = 64 // b
    c = min(b - 1, e)
    d = np.uint64(sum(1 << (j * (b - 1)) for j in range(c)))
    r = np.zeros_like(m)
    with np.errstate(over="ignore"):
        for k0 in range(0, e, c):
            r |= (((m >> np.uint64(k0)) & np.uint64((1 << c) - 1)) * d) << np.uint64(k0 * b)
    return (r << np.uint64(b - 1)) & np.uint64(top_bits(b))


def test_flag_deposit_places_every_pattern():
    rng = np.random.default_rng(0)
    for b in range(1, 33):
        e = 64 // b
        if e <= 21:
            pats = np.arange(1 << e, dtype=np.uint64)
        else:
            pats = rng.integers(0, 1 << 63, size=1 << 18, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
            pats &= np.uint64(M64 if e == 64 else (1 << e) - 1)
        # the expected word: bit k of the pattern on the top bit of field k
        want = np.zeros_like(pats)
        for k in range(e):
            want |= ((pats >> np.uint64(k)) & np.uint64(1)) << np.uint64(k * b + b - 1)
        assert np.array_equal(deposit(b, pats), want), b
        # bits of m above the E flags change nothing
        if e < 64:
            noisy = pats | (rng.integers(0, 1 << 63, size=pats.size, dtype=np.uint64) << np.uint64(e))
            assert np.array_equal(deposit(b, noisy), want), b
