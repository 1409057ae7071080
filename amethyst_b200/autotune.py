"""Autotuner for the launch knobs of the operator layer.

Every knob here changes only how work is laid out on the GPU (block shape, CTAs per SM, staging
depth, decode policy), never the integer results, so any candidate is a valid answer and the
tuner only compares times.  Candidates are timed with CUDA events on the current stream after a
warm-up, and the winner is remembered per (device, workload signature) in memory and, when a
cache path is given, in a small JSON file.

  tune_batch(cols, preds)        -> amx_batch_tuning for a batch of columns (threads, CTAs per SM,
                                    slab words per thread = the tile size)
  tune_pipeline(step, cands)     -> amx_tuning for single-column operators (policy, staging)
"""
from __future__ import annotations

import ctypes as C
import json
import os

import torch

from . import _capi as A

_cache: dict[str, dict] = {}


def _device_key() -> str:
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}/{p.multi_processor_count}"


def _load(path: str | None) -> None:
    if path and os.path.exists(path) and not _cache:
        try:
            _cache.update(json.load(open(path)))
        except (OSError, ValueError):
            pass


def _store(path: str | None) -> None:
    if path:
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def time_fn(fn, reps: int = 5, warmup: int = 2) -> float:
    """Mean milliseconds of fn() over `reps` calls, CUDA events on the current stream."""
    s = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def batch_signature(cols) -> str:
    """Workload signature of a batch: column count, total elements and the width histogram in
    8-bit buckets (the tile shape depends on the width)."""
    hist = [0, 0, 0, 0]
    total = 0
    for c in cols:
        hist[min(3, (c.bits - 1) // 8)] += 1
        total += c.n
    return f"batch/{len(cols)}/{total.bit_length()}/{hist}"


# (threads per CTA, CTAs per SM (0: as many as fit), slab words per thread: the tile size)
BATCH_CANDIDATES = [(256, 0, 8), (256, 0, 4), (256, 0, 2), (512, 0, 8), (512, 0, 4), (256, 1, 8)]


def tune_batch(cols, preds, candidates=BATCH_CANDIDATES, reps: int = 3, cache_path: str | None = None):
    """Times each (threads, CTAs per SM, words per thread) candidate on the batch itself; returns
    (best amx_batch_tuning, {candidate: ms})."""
    from .ops import Batch

    _load(cache_path)
    key = f"{_device_key()}/{batch_signature(cols)}"
    if key in _cache:
        t = _cache[key]["best"]
        return A.BatchTuning(t[0], t[1], t[2]), _cache[key]["times"]
    times = {}
    for thr, per_sm, wpt in candidates:
        tun = A.BatchTuning(thr, per_sm, wpt)
        b = Batch(cols, preds, tun)
        times[f"{thr}x{per_sm}x{wpt}"] = time_fn(b.run, reps=reps, warmup=1)
        del b
    best = min(times, key=times.get)
    thr, per_sm, wpt = (int(x) for x in best.split("x"))
    _cache[key] = {"best": [thr, per_sm, wpt], "times": times}
    _store(cache_path)
    return A.BatchTuning(thr, per_sm, wpt), times


PIPELINE_CANDIDATES = [
    # staged_bytes, compact_stages, policy (0 automatic, 1 generic)
    (0, 0, 0),
    (96 * 1024, 3, 0),
    (64 * 1024, 2, 0),
    (0, 0, 1),
]


def tune_pipeline(step, signature: str, candidates=PIPELINE_CANDIDATES, reps: int = 5,
                  cache_path: str | None = None):
    """Times `step()` (one call of a single-column operator) under each amx_tuning candidate;
    leaves the best one set for this thread and returns (amx_tuning, {candidate: ms})."""
    lib = A.lib()
    _load(cache_path)
    key = f"{_device_key()}/pipe/{signature}"
    if key in _cache:
        t = A.Tuning(*_cache[key]["best"], 0)
        A.check(lib.amx_set_tuning(C.byref(t)))
        return t, _cache[key]["times"]
    times = {}
    for sb, cs, pol in candidates:
        t = A.Tuning(sb, cs, pol, 0)
        A.check(lib.amx_set_tuning(C.byref(t)))
        times[f"{sb}/{cs}/{pol}"] = time_fn(step, reps=reps, warmup=2)
    best = min(times, key=times.get)
    sb, cs, pol = (int(x) for x in best.split("/"))
    t = A.Tuning(sb, cs, pol, 0)
    A.check(lib.amx_set_tuning(C.byref(t)))
    _cache[key] = {"best": [sb, cs, pol], "times": times}
    _store(cache_path)
    return t, times
