"""Seeded synthetic columns, on the GPU (amx_fill_uniform / amx_fill_from_cdf) and -- with the
same per-element function -- on the host in numpy, for workloads that must be built without a
GPU (the CPU baseline).

value(i) = top `bits` bits of xorshift64(splitmix64(seed + (i + 1) * 0x9E3779B97F4A7C15)).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def draws_np(seed: int, start: int, count: int) -> np.ndarray:
    i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
        z ^= z << np.uint64(13)
        z ^= z >> np.uint64(7)
        z ^= z << np.uint64(17)
    return z


def uniform_np(seed: int, bits: int, n: int, chunk: int = 1 << 24) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    for s in range(0, n, chunk):
        c = min(chunk, n - s)
        d = draws_np(seed, s, c)
        out[s:s + c] = d if bits >= 64 else (d >> np.uint64(64 - bits))
    return out


def zipf_cdf(groups: int, s: float) -> np.ndarray:
    w = 1.0 / np.arange(1, groups + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w) / w.sum()
    cdf[-1] = 1.0
    return cdf


def uniform_gpu(n: int, bits: int, seed: int, elem_bytes: int = 4, stream=None):
    import torch

    from ._capi import check, lib

    t = torch.empty(max(n, 4), dtype=torch.int32 if elem_bytes == 4 else torch.int64, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream()
    check(lib().amx_fill_uniform(C.c_void_p(t.data_ptr()), n, elem_bytes, bits, seed, C.c_void_p(s.cuda_stream)))
    return t


def keys_from_cdf_gpu(n: int, cdf: np.ndarray, seed: int, stream=None):
    import torch

    from ._capi import check, lib

    t = torch.empty(max(n, 4), dtype=torch.int32, device="cuda")
    d_cdf = torch.from_numpy(np.ascontiguousarray(cdf, dtype=np.float64)).cuda()
    s = stream if stream is not None else torch.cuda.current_stream()
    check(lib().amx_fill_from_cdf(C.c_void_p(t.data_ptr()), n, C.c_void_p(d_cdf.data_ptr()), len(cdf), seed,
                                  C.c_void_p(s.cuda_stream)))
    return t, d_cdf
