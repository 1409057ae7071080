"""Shared test helpers: input generation with dirty unused bits, and GPU <-> oracle plumbing."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

PLAIN32, PLAIN64, SLAB, NOGAPS = 0, 1, 2, 3
FORMATS = [PLAIN32, PLAIN64, SLAB, NOGAPS]


def valid_width(fmt, bits):
    return 1 <= bits <= (32 if fmt == PLAIN32 else 64)


def values(seed, bits, n):
    return O.uniform_values(seed, bits, n)


def dirty(raw: np.ndarray, fmt: int, bits: int, n: int, seed: int) -> np.ndarray:
    """Fill every bit that holds no element value with random garbage, as the reference's
    inputs do (random 64-bit words, src/main.cu:244-250).  Readers must ignore those bits."""
    rng = np.random.default_rng(seed)
    raw = raw.copy()
    nb = O.storage_bytes(fmt, bits, n)
    if nb == 0:
        return raw
    if fmt == PLAIN32:
        w = raw[:nb].view(np.uint32)
        if bits < 32:
            junk = rng.integers(0, 2**32, size=w.size, dtype=np.uint64).astype(np.uint32)
            w |= junk & np.uint32(~((1 << bits) - 1) & 0xFFFFFFFF)
    elif fmt == PLAIN64:
        w = raw[:nb].view(np.uint64)
        if bits < 64:
            junk = rng.integers(0, 2**63, size=w.size, dtype=np.uint64) * np.uint64(2)
            w |= junk & np.uint64(~((1 << bits) - 1) & 0xFFFFFFFFFFFFFFFF)
    elif fmt == SLAB:
        w = raw[:nb].view(np.uint64)
        eps = 64 // bits
        live = eps * bits
        if live < 64:
            junk = rng.integers(0, 2**63, size=w.size, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
            w |= junk & np.uint64(~((1 << live) - 1) & 0xFFFFFFFFFFFFFFFF)
        # fields past n in the last slab are unused too
        k = n % eps
        if k:
            junk = int(rng.integers(0, 2**63)) | 1
            unused_fields = ((1 << live) - 1) & ~((1 << (k * bits)) - 1)
            w[-1] |= np.uint64((junk << (k * bits)) & unused_fields & 0xFFFFFFFFFFFFFFFF)
    else:
        w = raw[:nb].view(np.uint64)
        tail = (n * bits) % 64
        if tail:
            junk = int(rng.integers(0, 2**63)) | 1
            w[-1] |= np.uint64((junk << tail) & 0xFFFFFFFFFFFFFFFF)
    return raw


def make_column(seed, fmt, bits, n, vals=None, dirty_bits=True):
    v = values(seed, bits, n) if vals is None else np.asarray(vals, dtype=np.uint64)
    raw = O.encode(fmt, bits, v)
    if dirty_bits:
        raw = dirty(raw, fmt, bits, n, seed + 7)
    return v, raw


def to_gpu(raw: np.ndarray, n, fmt, bits, device="cuda"):
    import torch

    from amethyst_b200.ops import PackedColumn

    col = PackedColumn.empty(n, fmt, bits, device)
    t = torch.from_numpy(raw.copy())
    m = min(t.numel(), col.data.numel())
    col.data[:m].copy_(t[:m])
    return col


def gpu_bytes(col, count=None) -> np.ndarray:
    nb = O.storage_bytes(col.fmt, col.bits, col.n if count is None else count)
    return col.data[:nb].cpu().numpy()


def mask_from_bytes(mask_u8: np.ndarray, n: int) -> np.ndarray:
    words = (n + 31) // 32
    buf = np.zeros(words * 4 + 16, dtype=np.uint8)
    buf[: min(len(mask_u8), words * 4)] = mask_u8[: words * 4]
    m = buf.view(np.uint32)[:words].copy()
    if n % 32:
        m[-1] &= np.uint32((1 << (n % 32)) - 1)
    return m
