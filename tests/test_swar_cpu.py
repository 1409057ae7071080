"""The single-multiplication flag gather of the field-parallel slab policy (swar_gather_flags in
amethyst_b200/csrc/amx_swar.cuh), checked exhaustively on the host: for every width B = 8..32 and
every pattern of the floor(64/B) field flags, (g * M) >> (E(B-1)) & (2^E - 1) equals the pattern;
at B = 7 it does not, so the kernel keeps the per-field loop below B = 8."""


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
