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


def sum_fits(b, spt):
    """swar_sum_fits<B, SPT>(): every two-field lane holds the sum of SPT fields."""
    need = b + spt.bit_length()
    for k in range(64 // b):
        room = 64 - k * b if k % 2 == 0 else 64 - (k - 1) * b
        if min(room, 2 * b) < need:
            return False
    return True


def test_field_parallel_masked_sum():
    """swar_masked_sum: whole-field masks from the flags by one product, even and odd fields summed
    in two-field lanes, against field-by-field sums of the passing fields (random words with junk
    padding bits, every flag pattern style), for every width whose lanes hold SPT sums."""
    rng = np.random.default_rng(3)
    fits = []
    for b in range(1, 33):
        e = 64 // b
        spt = 1 if e >= 64 else min(8, 64 // e)
        if not sum_fits(b, spt):
            continue
        fits.append(b)
        fm = (1 << b) - 1
        top = sum(1 << (k * b + b - 1) for k in range(e))
        even = sum(fm << (k * b) for k in range(0, e, 2))
        for trial in range(400):
            words = [int(w) for w in rng.integers(0, 1 << 63, size=spt, dtype=np.uint64) * 2 + 1]
            if trial % 3 == 0:  # every field at its maximum, junk above the fields
                words = [sum(fm << (k * b) for k in range(e)) | (w & ~((1 << (e * b)) - 1) & M64) for w in words]
            flags = [int(f) & top for f in rng.integers(0, 1 << 63, size=spt, dtype=np.uint64) * 2]
            if trial % 5 == 0:
                flags = [top] * spt
            a = bb = 0
            for x, g in zip(words, flags):
                m = x & (((g >> (b - 1)) * fm) & M64)
                a = (a + (m & even)) & M64
                bb = (bb + ((m >> b) & even)) & M64
            got = 0
            for k in range(0, e, 2):
                got += (a >> (k * b)) & ((1 << min(64 - k * b, 2 * b)) - 1)
                if k + 1 < e:
                    got += (bb >> (k * b)) & ((1 << min(64 - k * b, 2 * b)) - 1)
            want = sum((x >> (k * b)) & fm for x, g in zip(words, flags) for k in range(e) if (g >> (k * b + b - 1)) & 1)
            assert got == want, (b, trial)
    assert fits == [1, 2, 4, 5, 6, 8, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 22, 23, 24, 25, 26, 27, 28, 29, 30,
                    31, 32]


def test_bit_plane_sum():
    """swar_plane_sum: the passing fields' bits counted per bit position b and weighted by 2^b,
    against field-by-field sums, for the narrow widths up to 9 bits (the kernel takes it where the
    lanes do not fit at its run length: 3 bits, or 1-3 bits with runs of 8 slabs)."""
    rng = np.random.default_rng(4)
    for b in range(1, 10):
        e = 64 // b
        spt = 1 if e >= 64 else min(8, 64 // e)
        fm = (1 << b) - 1
        top = sum(1 << (k * b + b - 1) for k in range(e))
        low = sum(1 << (k * b) for k in range(e))
        for trial in range(300):
            words = [int(w) for w in rng.integers(0, 1 << 63, size=spt, dtype=np.uint64) * 2 + 1]
            if trial % 3 == 0:
                words = [sum(fm << (k * b) for k in range(e)) | (w & ~((1 << (e * b)) - 1) & M64) for w in words]
            flags = [int(f) & top for f in rng.integers(0, 1 << 63, size=spt, dtype=np.uint64) * 2]
            if trial % 5 == 0:
                flags = [top] * spt
            cnt = [0] * b
            for x, g in zip(words, flags):
                m = x & (((g >> (b - 1)) * fm) & M64)
                for p in range(b):
                    cnt[p] += bin(m & ((low << p) & M64)).count("1")
            got = sum(c << p for p, c in enumerate(cnt))
            want = sum((x >> (k * b)) & fm for x, g in zip(words, flags) for k in range(e) if (g >> (k * b + b - 1)) & 1)
            assert got == want, (b, trial)
