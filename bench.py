"""Benchmark of the Amethyst B200 operator layer.

Default workload (the operator-chain configuration, one step = one pass):
  A: 2^26 uint32 values uniform in [0, 2^7), packed in 7-bit slabs;
  B: 2^26 uint32 values uniform in [0, 2^13), packed in 13-bit slabs;
  C = A + B at 14 bits, keep C >= 2^13, compressstore the survivors as 14-bit slabs, and sum
  them into a uint64 -- one fused pass (amx_chain) through the C ABI.
`value` is packed GB/s = algorithmic bytes (packed inputs + packed output + scalars) / time,
with inputs resident in HBM (194.9 MB > 126 MB L2, so no flush is needed between steps).
`e2e` is the same metric through the same call with pinned host buffers, the host->device
copy of the inputs and the device->host copy of the results inside the timed region.

--impl reference runs the CPU arm: the scalar C oracle (a restatement of the reference's
accessors and operators; the reference itself has no CPU implementation of the path) on all
host cores over the same workload.

Multi-GPU (torchrun): every rank runs its own copy of the workload on its own GPU (the path
has no exchange step); value = all ranks' bytes / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "packed-op GB/s & % HBM peak; batched+learned-format vs plain, 1 B200, bit-exact"
N_CHAIN = 1 << 26
BITS_A, BITS_B, BITS_C = 7, 13, 14
THRESH = 1 << 13
SEED_A, SEED_B = 0x5EED_A, 0x5EED_B


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def storage_bytes(fmt, bits, n):
    if fmt == 0:
        return 4 * n
    if fmt == 1:
        return 8 * n
    if fmt == 2:
        eps = 64 // bits
        return 8 * ((n + eps - 1) // eps)
    return 8 * ((n * bits + 63) // 64)


# ------------------------------------------------------------------------------------------
# clocks during the timed region (NVML reads only)
# ------------------------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock"}

    def __init__(self, index):
        self.samples, self.reasons, self.stop_flag = [], 0, False
        self.ok = False
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None

    def _sample(self):
        try:
            self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            try:
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                r = self.nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
            self.reasons |= int(r) & ~0x1
        except Exception:
            pass

    def _run(self):
        while not self.stop_flag:
            self._sample()
            time.sleep(0.01)

    def start(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        if self.ok:
            self.stop_flag = True
            self.t.join()
            self._sample()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": [v for k, v in self.REASONS.items() if self.reasons & k], "samples": len(self.samples)}


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
def pack_gpu(n, bits, seed, fmt):
    """Generate uniform values on the GPU and encode them with amx_convert."""
    from amethyst_b200 import datagen, ops

    plain = datagen.uniform_gpu(n, bits, seed)
    src = ops.PackedColumn(plain.view(__import__("torch").uint8), n, 0, 32)
    return ops.convert(src, fmt, bits)


def time_steps(fn, steps, warmup, stream):
    """W warm-up calls, then exactly `steps` timed calls with an event pair around each one."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for a, b in evs:
        a.record(stream)
        fn()
        b.record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    per = [a.elapsed_time(b) for a, b in evs]
    return total_ms, per


def chain_workload(dev, out_fmt=2, a_fmt=2, b_fmt=2, thresh=THRESH):
    """Build the chain inputs and return (step function, algorithmic bytes fn, state)."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = N_CHAIN
    a = pack_gpu(n, BITS_A, SEED_A, a_fmt)
    b = pack_gpu(n, BITS_B, SEED_B, b_fmt)
    out = ops.PackedColumn.empty(n, out_fmt, BITS_C)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    agg = torch.zeros(2, dtype=torch.int64, device=dev)
    ws = ops.workspace(n)
    pred = ops.predicate(A.PRED_GE, thresh, 0, BITS_C)
    desc = A.ChainDesc(A.OP_ADD, BITS_C, pred, A.AGG_SUM, 0)
    import ctypes as C

    L = A.lib()
    a_d, b_d, o_d = a.desc, b.desc, out.desc
    args = (C.byref(desc), C.byref(a_d), C.byref(b_d), C.byref(o_d), None, C.c_void_p(cnt.data_ptr()),
            C.c_void_p(agg.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel())
    state = {"a": a, "b": b, "out": out, "cnt": cnt, "agg": agg, "ws": ws, "desc": desc, "n": n}

    def step(stream_ptr=None):
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream) if stream_ptr is None else stream_ptr
        A.check(L.amx_chain(*args, s))

    in_bytes = storage_bytes(a_fmt, BITS_A, n) + storage_bytes(b_fmt, BITS_B, n)

    def alg_bytes(count):
        return in_bytes + storage_bytes(out_fmt, BITS_C, count) + 16

    return step, alg_bytes, state, in_bytes


def e2e_chain(dev, steps, warmup):
    """amx_chain through the C ABI with pinned host buffers: H2D inputs, chain, D2H results."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A

    step, alg_bytes, st, in_bytes = chain_workload(dev)
    a, b, out = st["a"], st["b"], st["out"]
    ha = torch.empty(a.data.numel(), dtype=torch.uint8, pin_memory=True)
    hb = torch.empty(b.data.numel(), dtype=torch.uint8, pin_memory=True)
    ha.copy_(a.data)
    hb.copy_(b.data)
    hout = torch.empty(out.data.numel(), dtype=torch.uint8, pin_memory=True)
    hres = torch.empty(4, dtype=torch.int64, pin_memory=True)
    stream = torch.cuda.current_stream()
    d2h = [0]

    def e2e_step():
        a.data.copy_(ha, non_blocking=True)
        b.data.copy_(hb, non_blocking=True)
        step()
        hres[:2].copy_(st["cnt"], non_blocking=True)
        hres[2:].copy_(st["agg"], non_blocking=True)
        stream.synchronize()
        c = int(hres[0])
        nb = storage_bytes(2, BITS_C, c)
        hout[:nb].copy_(out.data[:nb], non_blocking=True)
        stream.synchronize()
        d2h[0] = nb + 16

    for _ in range(warmup):
        e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        e2e_step()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    c = int(hres[0])
    return {"value": alg_bytes(c) / dt / 1e9, "unit": "GB/s", "h2d_bytes_per_step": in_bytes,
            "d2h_bytes_per_step": d2h[0], "ms_per_step": dt * 1e3}


def fc_1gib(dev, steps, warmup):
    """The north-star column: 1 GiB of 11-bit slabs (2^27 slabs, 671,088,640 elements),
    fused filter v < 205 + compressstore into 11-bit slabs."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = (1 << 27) * 5
    col = pack_gpu(n, 11, 0xC0FFEE, 2)
    out = ops.PackedColumn.empty(n, 2, 11)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    ws = ops.workspace(n)
    pred = ops.predicate(A.PRED_LT, 205, 0, 11)
    L = A.lib()
    cd, od = col.desc, out.desc

    def step():
        A.check(L.amx_filter_compressstore(C.byref(cd), C.byref(pred), C.byref(od), C.c_void_p(cnt.data_ptr()),
                                           C.c_void_p(ws.data_ptr()), ws.numel(),
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream)))

    total, per = time_steps(step, steps, warmup, torch.cuda.current_stream())
    c = int(cnt[0].item())
    byts = storage_bytes(2, 11, n) + storage_bytes(2, 11, c) + 8
    ms = total / steps
    res = {"workload": "filter v<205 + compressstore, 1 GiB column of 11-bit slabs (671,088,640 elements)",
           "GB_s": byts / (ms * 1e-3) / 1e9, "ms_per_step": ms, "selectivity": c / n, "alg_bytes": byts}
    # the same column through the other two single-column operators: filter to a bitmask, and
    # count + sum of the passing values
    mask = torch.empty(ops.mask_words(n) + 4, dtype=torch.int32, device=dev)
    agg = torch.zeros(2, dtype=torch.int64, device=dev)
    desc = A.ChainDesc(A.OP_LHS, 11, pred, A.AGG_SUM, 0)
    sp = lambda: C.c_void_p(torch.cuda.current_stream().cuda_stream)  # noqa: E731
    for name, fn, extra_bytes in [
        ("filter_to_bitmask", lambda: A.check(L.amx_filter(C.byref(cd), C.byref(pred), C.c_void_p(mask.data_ptr()),
                                                           C.c_void_p(ws.data_ptr()), ws.numel(), sp())),
         4 * ((n + 31) // 32)),
        ("count_and_sum", lambda: A.check(L.amx_chain(C.byref(desc), C.byref(cd), None, None, None,
                                                      C.c_void_p(cnt.data_ptr()), C.c_void_p(agg.data_ptr()),
                                                      C.c_void_p(ws.data_ptr()), ws.numel(), sp())), 16)]:
        t2, _ = time_steps(fn, steps, warmup, torch.cuda.current_stream())
        ms2 = t2 / steps
        b2 = storage_bytes(2, 11, n) + extra_bytes
        res[name] = {"GB_s": round(b2 / (ms2 * 1e-3) / 1e9, 2), "ms_per_step": round(ms2, 5), "alg_bytes": b2}
    del col, out, ws, mask
    torch.cuda.empty_cache()
    return res


def batched_512(dev, steps):
    """512 slab columns, lengths log-uniform in [2^12, 2^24], widths uniform in 1..32, values
    uniform in [0, 2^w), thresholds v < T drawn for selectivity uniform in [0.01, 0.99]:
    filter + compressstore + sum of every column in one persistent launch replayed from a CUDA
    graph (block shape from the autotuner), against 512 sequential single-column launches."""
    import ctypes as C

    import numpy as np
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import autotune, ops

    rng = np.random.default_rng(0xBA7C4)
    ncols = 512
    ns = np.exp(rng.uniform(np.log(2 ** 12), np.log(2 ** 24), ncols)).astype(np.int64)
    widths = rng.integers(1, 33, ncols)
    sel = rng.uniform(0.01, 0.99, ncols)
    cols, preds = [], []
    for i in range(ncols):
        n, w = int(ns[i]), int(widths[i])
        cols.append(pack_gpu(n, w, 0xC010 + i, 2))
        preds.append(ops.predicate(A.PRED_LT, max(1, int(round(sel[i] * (1 << w)))), 0, w))
    torch.cuda.synchronize()
    tuning, tune_times = autotune.tune_batch(cols, preds)
    b = ops.Batch(cols, preds, tuning)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.run(s)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(s)
    reps = max(3, min(steps, 20))
    stream = torch.cuda.current_stream()
    tot, _ = time_steps(g.replay, reps, 3, stream)
    ms_b = tot / reps
    counts = b.counts.cpu().numpy().view(np.uint64).copy()
    sums = b.sums.cpu().numpy().view(np.uint64).copy()

    # the same work as 512 sequential single-column launches (fused chain per column)
    L = A.lib()
    outs = b.outs
    cnt = torch.zeros(2 * ncols, dtype=torch.int64, device=dev)
    agg = torch.zeros(2 * ncols, dtype=torch.int64, device=dev)
    ws = ops.workspace(int(ns.max()))
    descs = [A.ChainDesc(A.OP_LHS, int(widths[i]), preds[i], A.AGG_SUM, 0) for i in range(ncols)]
    cds = [c.desc for c in cols]
    ods = [o.desc for o in outs]

    def seq():
        sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for i in range(ncols):
            A.check(L.amx_chain(C.byref(descs[i]), C.byref(cds[i]), None, C.byref(ods[i]), None,
                                C.c_void_p(cnt.data_ptr() + 16 * i), C.c_void_p(agg.data_ptr() + 16 * i),
                                C.c_void_p(ws.data_ptr()), ws.numel(), sp))

    tot2, _ = time_steps(seq, reps, 2, stream)
    ms_s = tot2 / reps
    sc = cnt.cpu().numpy().view(np.uint64)[0::2]
    sa = agg.cpu().numpy().view(np.uint64)[0::2]
    same = bool(np.array_equal(sc, counts) and np.array_equal(sa, sums))
    in_bytes = sum(storage_bytes(2, int(widths[i]), int(ns[i])) for i in range(ncols))
    out_bytes = sum(storage_bytes(2, int(widths[i]), int(counts[i])) for i in range(ncols))
    byts = in_bytes + out_bytes + 16 * ncols
    res = {"workload": "512 slab columns, n log-uniform [2^12, 2^24], widths 1..32, selectivity U[0.01, 0.99]: "
                       "filter + compressstore + sum",
           "elements": int(ns.sum()), "alg_bytes": byts,
           "batched_graph": {"ms": round(ms_b, 4), "GB_s": round(byts / (ms_b * 1e-3) / 1e9, 2),
                             "tuning": {"threads": tuning.threads, "ctas_per_sm": tuning.ctas_per_sm,
                                        "words_per_thread": tuning.words_per_thread},
                             "autotune_ms": {k: round(v, 4) for k, v in tune_times.items()}},
           "sequential_512_launches": {"ms": round(ms_s, 4), "GB_s": round(byts / (ms_s * 1e-3) / 1e9, 2)},
           "speedup": round(ms_s / ms_b, 3), "results_equal": same}
    del g, b, cols, outs
    torch.cuda.empty_cache()
    return res


def matmul_4096(dev, steps):
    """Dense 4096 x 4096 times 4096 x 4096 over unsigned 7-bit entries in slab rows (9 per slab,
    456 slabs per row), integer tensor cores with exact int32 accumulation, output packed at the
    narrowest width holding the largest entry.  One step = one amx_matmul call (the default
    two-pass path: unpack, GEMM, pack); the fused kernel (amx_tuning.policy 2: unpack in shared
    memory, pack from the accumulators) is timed beside it and its output compared byte for
    byte."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import datagen, ops

    M = N = K = 4096

    def slab_matrix(rows, cols, bits, seed):
        eps = 64 // bits
        rs = (cols + eps - 1) // eps
        plain = datagen.uniform_gpu(rows * cols, bits, seed).view(rows, cols)
        pad = torch.zeros(rows, rs * eps, dtype=torch.int32, device=dev)
        pad[:, :cols] = plain
        flat = ops.PackedColumn(pad.reshape(-1).contiguous().view(torch.uint8), rows * rs * eps, 0, 32)
        col = ops.convert(flat, A.SLAB, bits)
        return ops.PackedColumn(col.data, rows * cols, A.SLAB, bits)

    a = slab_matrix(M, K, 7, 0xA11)
    b = slab_matrix(K, N, 7, 0xB22)
    ws = ops.matmul_workspace(M, N, K)
    out, width = ops.matmul(a, b, M, N, K, ws=ws)
    L = A.lib()

    def step():
        A.check(L.amx_matmul(C.byref(a.desc), C.byref(b.desc), M, N, K, C.byref(out.desc),
                             C.c_void_p(width.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream)))

    reps = max(3, min(steps, 30))
    tot, _ = time_steps(step, reps, 3, torch.cuda.current_stream())
    ms = tot / reps
    A.check(L.amx_matmul_status(C.c_void_p(ws.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    bits = int(width[0].item())
    nb = M * ((N + 64 // bits - 1) // (64 // bits)) * 8  # slab rows padded to whole words
    two_pass = out.data[:nb].clone()
    # the fused kernel (operands unpacked in shared memory from TMA-staged packed slices, the
    # product packed from the tensor-memory accumulators), for comparison
    A.check(L.amx_set_tuning(C.byref(A.Tuning(0, 0, 2, 0))))
    try:
        tot2, _ = time_steps(step, reps, 3, torch.cuda.current_stream())
        torch.cuda.synchronize()
        same = bool(torch.equal(two_pass, out.data[:nb])) and int(width[0].item()) == bits
    finally:
        A.check(L.amx_set_tuning(None))
    ms2 = tot2 / reps
    res = {"workload": "4096^3 u7 x u7 slab matrices -> narrowest-width slabs; default: u8 operands unpacked once "
                       "to the workspace, int32 product packed by a second pass",
           "ms_per_step": round(ms, 4), "TOPS": round(2 * M * N * K / (ms * 1e-3) / 1e12, 1), "out_bits": bits,
           "fused_ms": round(ms2, 4), "fused_TOPS": round(2 * M * N * K / (ms2 * 1e-3) / 1e12, 1),
           "identical": same}
    del a, b, ws, out, two_pass
    torch.cuda.empty_cache()
    return res


def fc_cfg1(dev, steps):
    """The plain filter+compressstore configuration: 2^24 uint32 values uniform in [0, 2^11) in
    11-bit slabs (26.8 MB, smaller than L2), predicate v < 205, output in 11-bit slabs.  L2 is
    flushed (a 256 MB buffer rewritten) before every timed call, outside its event pair."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 1 << 24
    col = pack_gpu(n, 11, 0xC0FFEE, 2)
    out = ops.PackedColumn.empty(n, 2, 11)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    ws = ops.workspace(n)
    pred = ops.predicate(A.PRED_LT, 205, 0, 11)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    L = A.lib()
    cd, od = col.desc, out.desc
    stream = torch.cuda.current_stream()

    def step():
        A.check(L.amx_filter_compressstore(C.byref(cd), C.byref(pred), C.byref(od), C.c_void_p(cnt.data_ptr()),
                                           C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(stream.cuda_stream)))

    for _ in range(3):
        step()
    reps = max(3, min(steps, 30))
    ms = 0.0
    for _ in range(reps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= reps
    c = int(cnt[0].item())
    byts = storage_bytes(2, 11, n) + storage_bytes(2, 11, c) + 8
    del col, out, ws, flush
    torch.cuda.empty_cache()
    return {"workload": "filter v<205 + compressstore, 2^24 elements in 11-bit slabs (26.8 MB), L2 flushed per call",
            "GB_s": round(byts / (ms * 1e-3) / 1e9, 2), "ms_per_step": round(ms, 5), "selectivity": c / n,
            "alg_bytes": byts}


def groupby_wide(dev, steps):
    """Group-by with 32-bit keys, hash tables (amx_groupby) against radix sort + reduce-by-key
    (amx_groupby_sort), 2^26 keys in 32-bit slabs and 2^26 u16 values in 16-bit slabs: Zipf(1.1)
    draws from 100,000 random keys; uniform draws from 2^20 and from 2^23 random keys; uniform
    32-bit keys (about 2^26 distinct groups).  The two outputs are compared byte for byte."""
    import ctypes as C

    import numpy as np
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import datagen, ops

    n = 1 << 26
    L = A.lib()
    vals = pack_gpu(n, 16, 0x7A2, 2)
    rows = {}
    for name in ("zipf_100k_keys", "uniform_from_1m_keys", "uniform_from_8m_keys", "uniform_32bit_keys"):
        if name == "zipf_100k_keys":
            idx, _ = datagen.keys_from_cdf_gpu(n, datagen.zipf_cdf(100000, 1.1), 5)
            pool = torch.from_numpy(np.random.default_rng(6).choice(1 << 32, size=100000, replace=False)).to(dev)
            k32 = pool[idx[:n].long()].bitwise_and(0xFFFFFFFF).to(torch.int32)
            del idx, pool
            cap = 1 << 17
        elif name.startswith("uniform_from"):
            m = (1 << 20) if "1m" in name else (1 << 23)
            pool = torch.from_numpy(np.random.default_rng(7).choice(1 << 32, size=m, replace=False)).to(dev)
            idx = datagen.uniform_gpu(n, 32, 0x5EEE + m).long().bitwise_and(0xFFFFFFFF) % m
            k32 = pool[idx[:n]].bitwise_and(0xFFFFFFFF).to(torch.int32)
            del idx, pool
            cap = m
        else:
            k32 = datagen.uniform_gpu(n, 32, 0x5EED)
            cap = n
        keys = ops.convert(ops.PackedColumn(k32.contiguous().view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, 32)
        del k32
        torch.cuda.empty_cache()
        reps = max(3, min(steps, 10))
        gws = ops.groupby_workspace(32, cap)
        res = {}
        tot, _ = time_steps(lambda: res.__setitem__("h", ops.groupby(keys, vals, ws=gws, max_groups=cap)), reps, 3,
                            torch.cuda.current_stream())
        ms_h = tot / reps
        ops.groupby_status(gws, 32)
        del gws
        torch.cuda.empty_cache()
        sws = ops.aligned_bytes(int(L.amx_groupby_sort_workspace_bytes(n, 32, 16)), 256)
        tot, _ = time_steps(lambda: res.__setitem__("s", ops.groupby_sort(keys, vals, ws=sws, max_groups=cap)), reps,
                            3, torch.cuda.current_stream())
        ms_s = tot / reps
        A.check(L.amx_groupby_sort_status(C.c_void_p(sws.data_ptr()),
                                          C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        g = int(res["h"][3][0].item())
        same = g == int(res["s"][3][0].item())
        for x, y in zip(res["h"][:3], res["s"][:3]):
            nb = storage_bytes(x.fmt, x.bits, g)
            same = same and bool(torch.equal(x.data[:nb], y.data[:nb]))
        rows[name] = {"groups": g, "hash_ms": round(ms_h, 4), "sort_ms": round(ms_s, 4), "identical": same}
        del keys, sws, res
        torch.cuda.empty_cache()
    del vals
    torch.cuda.empty_cache()
    return {"workload": "group-by sum+count, 2^26 32-bit keys (32-bit slabs) + u16 values: hash tables vs radix "
                        "sort + reduce-by-key", "rows": rows}


def groupby_2e28(dev, steps):
    """Group-by at 1 GB: 2^28 keys Zipf(s=1.1) over 1000 groups packed at 10 bits, 2^28 values
    uniform in [0, 2^16) packed at 16 bits; per-group uint64 sum and count."""
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import datagen, ops

    n = 1 << 28
    cdf = datagen.zipf_cdf(1000, 1.1)
    keys32, _ = datagen.keys_from_cdf_gpu(n, cdf, 0x21F)
    keys = ops.convert(ops.PackedColumn(keys32.view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, 10)
    del keys32
    vals = pack_gpu(n, 16, 0x7A1, 2)
    torch.cuda.empty_cache()
    gws = torch.empty(int(A.lib().amx_groupby_workspace_bytes(10)) + 256, dtype=torch.uint8, device=dev)
    gws = gws[(-gws.data_ptr()) % 256:]
    res = {}

    def step():
        res["r"] = ops.groupby(keys, vals, ws=gws)

    reps = max(3, min(steps, 20))
    tot, _ = time_steps(step, reps, 3, torch.cuda.current_stream())
    ms = tot / reps
    ok, osum, ocnt, ng = res["r"]
    byts = keys.nbytes + vals.nbytes + int(ng[0].item()) * 24
    out = {"workload": "group-by sum+count: 2^28 Zipf(1.1) keys over 1000 groups at 10 bits, 2^28 u16 values",
           "ms_per_step": round(ms, 4), "GB_s": round(byts / (ms * 1e-3) / 1e9, 2), "groups": int(ng[0].item()),
           "alg_bytes": byts}
    del keys, vals, gws, res
    torch.cuda.empty_cache()
    return out


def cluster_mask(n, sel, clusters, dev):
    """`clusters` runs of floor(floor(sel * n) / clusters) set bits, run i starting at element
    i * floor(n / clusters) -- the reference's clustered compressstore masks
    (src/main.cu:59-101, modes 1 and 2 with 1 and 8 clusters) -- as LSB-first uint32 words."""
    import torch

    words = (n + 31) // 32
    m = torch.zeros(words + 4, dtype=torch.int64, device=dev)
    run = int(sel * n) // clusters
    for i in range(clusters):
        a = i * (n // clusters)
        b = a + run
        wa, wb = (a + 31) // 32, b // 32
        if wa < wb:
            m[wa:wb] = 0xFFFFFFFF
        for e0, e1 in ((a, min(b, wa * 32)), (max(a, wb * 32), b)):
            if e0 < e1:
                w = e0 // 32
                bits = ((1 << (e1 - w * 32)) - 1) & ~((1 << (e0 - w * 32)) - 1)
                m[w] |= bits
    return m.to(torch.int32)


def sums_671m(dev, steps):
    """Sum of every value of a 671,088,640-element slab column (amx_reduce, no predicate, no mask)
    at several widths: the automatic choice (field-parallel kernels where they apply) against the
    compile-time-width policy forced through amx_tuning.policy, results compared."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    L = A.lib()
    stream = torch.cuda.current_stream()
    s = C.c_void_p(stream.cuda_stream)
    n = 671088640
    k = max(3, min(steps, 20))
    res = torch.zeros(2, dtype=torch.int64, device=dev)
    rows = {}
    try:
        for bits in (1, 3, 4, 7, 8, 11, 16, 32):
            col = pack_gpu(n, bits, 0x5A + bits, 2)
            ws = ops.workspace(n)
            out = {}
            for name, pol in (("auto", 0), ("compile_time", 1 + bits)):
                A.check(L.amx_set_tuning(C.byref(A.Tuning(0, 0, pol, 0))) if pol else L.amx_set_tuning(None))

                def step():
                    A.check(L.amx_reduce(A.AGG_SUM, C.byref(col.desc), None, C.c_void_p(res.data_ptr()),
                                         C.c_void_p(ws.data_ptr()), ws.numel(), s))

                tot, _ = time_steps(step, k, 3, stream)
                out[name] = (tot / k, int(res[0].item()))
            A.check(L.amx_set_tuning(None))
            ms = out["auto"][0]
            rows[f"{bits}_bit"] = {"ms": round(ms, 4), "compile_time_ms": round(out["compile_time"][0], 4),
                                   "GB_s": round(col.nbytes / (ms * 1e-3) / 1e9, 1),
                                   "identical": out["auto"][1] == out["compile_time"][1]}
            del col, ws
            torch.cuda.empty_cache()
    finally:
        A.check(L.amx_set_tuning(None))
    return {"workload": "sum of a 671,088,640-element slab column, automatic kernel vs compile-time-width policy",
            "rows": rows}


def compressstore_masks(dev, steps):
    """compressstore of 2^27 elements in 11-bit slabs by a given mask, for the reference's mask
    distributions (src/main.cu:33-108, run.sh:6-22): uniform random bits, one cluster, eight
    clusters, at selectivities 0.01, 0.1, 0.5 and 0.9; output in 11-bit slabs.  Bytes = packed
    input + mask + packed output."""
    import ctypes as C

    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    n = 1 << 27
    col = pack_gpu(n, 11, 0x3A5C, 2)
    out = ops.PackedColumn.empty(n, 2, 11)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    ws = ops.workspace(n)
    r16 = pack_gpu(n, 16, 0x3A5D, 0)  # independent uniform 16-bit draws for the uniform masks
    L = A.lib()
    stream = torch.cuda.current_stream()
    rows = {}
    for sel in (0.01, 0.1, 0.5, 0.9):
        for name, clusters in (("uniform", 0), ("single_cluster", 1), ("multi_cluster_8", 8)):
            if clusters:
                mask = cluster_mask(n, sel, clusters, dev)
            else:
                mask = ops.filter(r16, ops.predicate(A.PRED_LT, int(round(sel * 65536))), ws=ws)

            def step():
                A.check(L.amx_compressstore(C.byref(col.desc), C.c_void_p(mask.data_ptr()), C.byref(out.desc),
                                            C.c_void_p(cnt.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
                                            C.c_void_p(stream.cuda_stream)))

            reps = max(3, min(steps, 20))
            tot, _ = time_steps(step, reps, 3, stream)
            ms = tot / reps
            c = int(cnt[0].item())
            byts = storage_bytes(2, 11, n) + 4 * ((n + 31) // 32) + storage_bytes(2, 11, c)
            rows[f"{name}_{sel}"] = {"ms": round(ms, 4), "GB_s": round(byts / (ms * 1e-3) / 1e9, 1),
                                     "selectivity": round(c / n, 5)}
            del mask
    del col, out, ws, r16
    torch.cuda.empty_cache()
    return {"workload": "compressstore by a given mask, 2^27 elements in 11-bit slabs -> 11-bit slabs", "rows": rows}


def mixed_chain(dev, steps, chains=64, lanes=8, exhaustive=True):
    """The mixed-chain workload: `chains` held-out synthetic operator chains (2..5 operators from
    {filter, compressstore, add, sub, mul, sum, min, max, group-by}, n log-uniform in [2^16,
    2^26], widths 1..32; those with at least one decision point), end to end with the inputs
    resident in HBM and every scalar result (aggregates, survivor counts, group counts) read back
    to the host, in two forms:
      plain     per column and per operator through the single-operator C ABI, every
                intermediate in slabs at its natural width, survivor counts read back after
                each compressstore to size the next call;
      batched   every chain an amx_program with the selector's storage formats, widths and
                kernel variants, all programs in one CUDA graph over `lanes` streams, one
                replay and one copy of all results.
    Regret: each chain's selector pick against the exhaustive best, both timed as replayed
    graphs of that chain alone.  Every form's results are compared bit for bit."""
    import numpy as np
    import torch

    from amethyst_b200 import chains as X
    from amethyst_b200 import ops
    from amethyst_b200 import selector as S

    rng = np.random.default_rng(99)
    specs, k = [], 0
    while len(specs) < chains:
        ch = X.random_chain(rng, seed=100000 + k)
        k += 1
        if X.decision_points(ch):
            specs.append(ch)
    results = torch.zeros(sum(len(c.ops) for c in specs), dtype=torch.int64, device=dev)
    runners, slot = [], 0
    for ch in specs:
        runners.append(S.ChainRunner(ch, results, slot))
        slot += len(ch.ops)
    sel = S.Selector.load()
    picks = sel.choices(runners)
    progs = [r.program(X.from_combo(p))[0] for r, p in zip(runners, picks)]
    graph = ops.Graph(progs, lanes=lanes)
    slab_progs = [r.program(X.fixed(X.DEFAULT_CHOICE))[0] for r in runners]
    slab_graph = ops.Graph(slab_progs, lanes=lanes)
    host = torch.empty(results.numel(), dtype=torch.int64, pin_memory=True)
    stream = torch.cuda.current_stream()

    def plain_step():
        for r in runners:
            r.run_plain()
        host.copy_(results, non_blocking=True)
        stream.synchronize()

    def graph_step(g):
        g.launch(stream)
        host.copy_(results, non_blocking=True)
        stream.synchronize()

    # bit-exactness: the plain form, the batched selector graph, the fixed-slab graph
    def digests(final_of):
        return [r.digest(final_of(i)) for i, r in enumerate(runners)]

    results.zero_()
    finals = [r.run_plain() for r in runners]
    torch.cuda.synchronize()
    ref = digests(lambda i: runners[i].plain_final_column(finals[i]))
    results.zero_()
    graph_step(graph)
    exact = digests(lambda i: runners[i].final_column(progs[i])) == ref
    results.zero_()
    graph_step(slab_graph)
    exact_slab = digests(lambda i: runners[i].final_column(slab_progs[i])) == ref

    reps = max(3, min(steps, 10))
    timings = {}
    for name, fn in [("plain", plain_step), ("batched", lambda: graph_step(graph)),
                     ("batched_fixed_slab", lambda: graph_step(slab_graph))]:
        for _ in range(2):
            fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        timings[name] = statistics.median(ts)
    res = {"workload": f"{len(specs)} held-out operator chains (2-5 operators, n log-uniform [2^16, 2^26], "
                       "widths 1..32), inputs resident, scalar results to the host",
           "chains": len(specs), "elements": int(sum(c.n for c in specs)), "lanes": lanes,
           "plain_ms": round(timings["plain"], 3), "batched_ms": round(timings["batched"], 3),
           "batched_fixed_slab_ms": round(timings["batched_fixed_slab"], 3),
           "speedup_e2e": round(timings["plain"] / timings["batched"], 3),
           "speedup_selector_in_graph": round(timings["batched_fixed_slab"] / timings["batched"], 3),
           "all_exact": bool(exact and exact_slab), "picks_histogram": np.bincount(
               [c for p in picks for c in p], minlength=X.K).tolist()}
    if exhaustive:
        regrets, combos = [], 0
        for r, p in zip(runners, picks):
            best, bc, table = S.exhaustive(r.chain, r, reps=3)
            combos += len(table)
            regrets.append(table[tuple(p)] / best - 1.0)
        res["regret"] = {"median": round(float(np.median(regrets)), 4), "mean": round(float(np.mean(regrets)), 4),
                         "p90": round(float(np.percentile(regrets, 90)), 4), "combinations_timed": combos}
    del graph, slab_graph, progs, slab_progs, runners
    torch.cuda.empty_cache()
    return res


def cpu_baseline_chain(st, threads):
    """The C oracle (scalar restatement of the reference semantics) on the host cores over the
    same packed inputs: the whole chain -- survivors compacted into 14-bit slabs, count and sum;
    also checks the GPU result (count, sum and the compacted bytes)."""
    import numpy as np

    from oracle import oracle as O

    n = st["n"]
    araw = st["a"].data.cpu().numpy()
    braw = st["b"].data.cpu().numpy()
    p = O.pred(4, THRESH)
    t0 = time.perf_counter()
    out, cnt, agg = O.chain_compress_mt(0, (araw, 2, BITS_A), (braw, 2, BITS_B), BITS_C, p, 0, 2, BITS_C, n, threads)
    dt = time.perf_counter() - t0
    gc = int(st["cnt"][0].item())
    ga = int(st["agg"].cpu().numpy().view(np.uint64)[0])
    same = gc == cnt and ga == agg and np.array_equal(st["out"].data[: len(out)].cpu().numpy(), out)
    in_bytes = storage_bytes(2, BITS_A, n) + storage_bytes(2, BITS_B, n)
    return dt, cnt, agg, same, in_bytes


def job_time_ms(local_ms, dist=None, device=None):
    """Whole-job time: the maximum of every rank's own device-timed total.  Every rank calls it
    after its timed region; the barrier first keeps a rank from reading before all have
    finished."""
    if dist is None:
        return float(local_ms)
    import torch

    dist.barrier()
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, bytes_per_rank, ms_per_step):
    """Aggregate packed GB/s of the job: every rank processes its own copy of the workload per
    step (replicas, weak scaling), so the job moves world x bytes_per_rank per step."""
    return world * bytes_per_rank / (ms_per_step * 1e-3) / 1e9


def run_gpu(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from amethyst_b200 import build as B

    if not os.path.exists(B.LIB):
        B.build()

    step, alg_bytes, st, in_bytes = chain_workload(dev)
    stream = torch.cuda.current_stream()
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    total_ms, per = time_steps(step, args.steps, 0, stream)
    sampler.stop()
    torch.cuda.synchronize()
    total_ms = job_time_ms(total_ms, dist, dev)
    count = int(st["cnt"][0].item())
    ms = total_ms / args.steps
    byts = alg_bytes(count)
    value = job_value(world, byts, ms)
    peak, peak_kind = measured_peaks()
    kern_ms = statistics.mean(per)
    achieved = byts / (kern_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get("chain_7_13_to_14_slab")

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "operator chain at 256 MB: A u7 slab + B u13 slab -> C 14 bits, filter C >= 2^13, "
                               "compressstore to 14-bit slabs, sum to uint64 (one fused pass)",
                   "elements": N_CHAIN, "input_bytes": in_bytes, "survivors": count,
                   "selectivity": count / N_CHAIN, "l2": "inputs (194.9 MB) larger than L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "hbm_frac": round(byts / (ms * 1e-3) / 1e9 / peak, 4),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                     "kernel": "amx::pipe_kernel<Slab2Pol<7,13,true,AMX_OP_ADD>>", "alg_bytes_per_launch": byts,
                     "launch_ms": round(kern_ms, 5)},
        "gpu_launches": args.steps,
        "clocks": sampler.summary(),
    }
    if rank == 0:
        # end to end through the same C ABI call with host buffers
        line["e2e"] = e2e_chain(dev, steps=max(3, min(args.steps, 20)), warmup=2)
        if world == 1 and not args.no_extra:
            extra = {}
            try:
                extra["fc_1gib"] = fc_1gib(dev, steps=max(3, min(args.steps, 30)), warmup=3)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["fc_1gib"] = {"error": str(e)}
            try:
                extra["fc_cfg1"] = fc_cfg1(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["fc_cfg1"] = {"error": str(e)}
            try:
                extra["groupby_2e28"] = groupby_2e28(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["groupby_2e28"] = {"error": str(e)}
            try:
                extra["groupby_wide"] = groupby_wide(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["groupby_wide"] = {"error": str(e)}
            try:
                extra["matmul_4096"] = matmul_4096(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["matmul_4096"] = {"error": str(e)}
            try:
                extra["batched_512"] = batched_512(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["batched_512"] = {"error": str(e)}
            try:
                extra["sums_671m"] = sums_671m(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["sums_671m"] = {"error": str(e)}
            try:
                extra["compressstore_masks"] = compressstore_masks(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["compressstore_masks"] = {"error": str(e)}
            try:
                extra["mixed_chain"] = mixed_chain(dev, args.steps)
            except Exception as e:  # pragma: no cover - reported, not fatal
                extra["mixed_chain"] = {"error": str(e)}
            for name, kw in [("chain_50pct", {"thresh": 4160}), ("chain_plain32_in", {"a_fmt": 0, "b_fmt": 0}),
                             ("chain_plain32_out", {"out_fmt": 0}),
                             ("chain_plain32_in_out", {"a_fmt": 0, "b_fmt": 0, "out_fmt": 0})]:
                s2, ab2, st2, ib2 = chain_workload(dev, **kw)
                tot2, per2 = time_steps(s2, max(3, min(args.steps, 50)), 3, stream)
                c2 = int(st2["cnt"][0].item())
                ms2 = tot2 / max(3, min(args.steps, 50))
                extra[name] = {"GB_s": round(ab2(c2) / (ms2 * 1e-3) / 1e9, 2), "ms_per_step": round(ms2, 5),
                               "selectivity": c2 / N_CHAIN, "alg_bytes": ab2(c2)}
                del s2, st2
            line["extra"] = extra
        if world == 1:
            threads = len(os.sched_getaffinity(0))
            dt, ccnt, cagg, ok, ib = cpu_baseline_chain(st, threads)
            line["cpu_baseline"] = {"value": round((ib + storage_bytes(2, BITS_C, ccnt) + 16) / dt / 1e9, 3),
                                    "unit": "GB/s", "cores": threads, "kind": "port",
                                    "sample": "the full chain workload once (compacted 14-bit slabs, count and sum; "
                                              "the C oracle)",
                                    "seconds": round(dt, 3), "matches_gpu": ok}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------------------------------
# reference (CPU) arm
# ------------------------------------------------------------------------------------------
def run_reference(args):
    import numpy as np

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from amethyst_b200 import datagen
    from oracle import oracle as O

    n = N_CHAIN
    a = O.encode(2, BITS_A, datagen.uniform_np(SEED_A, BITS_A, n))
    b = O.encode(2, BITS_B, datagen.uniform_np(SEED_B, BITS_B, n))
    threads = len(os.sched_getaffinity(0))
    p = O.pred(4, THRESH)
    steps = args.steps
    for _ in range(max(1, args.warmup)):
        O.chain_compress_mt(0, (a, 2, BITS_A), (b, 2, BITS_B), BITS_C, p, 0, 2, BITS_C, n, threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        _, cnt, agg = O.chain_compress_mt(0, (a, 2, BITS_A), (b, 2, BITS_B), BITS_C, p, 0, 2, BITS_C, n, threads)
    dt = (time.perf_counter() - t0) / steps
    byts = storage_bytes(2, BITS_A, n) + storage_bytes(2, BITS_B, n) + storage_bytes(2, BITS_C, cnt) + 16
    v = byts / dt / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "operator chain at 256 MB: A u7 slab + B u13 slab -> C 14 bits, filter C >= 2^13, "
                                   "compressstore to 14-bit slabs, sum to uint64", "elements": n, "survivors": cnt},
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                             "sample": "the full chain workload per step (survivors compacted into "
                                       "14-bit slabs, count and sum; the C oracle, which restates the reference's "
                                       "accessors and operators)"},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="amethyst", choices=["amethyst", "reference"])
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--only", default=None, help="run one secondary workload by name and print it")
    ap.add_argument("--lanes", type=int, default=8, help="streams of the mixed-chain graph (--only mixed_chain)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        import torch

        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        fn = {"mixed_chain": lambda d, k: mixed_chain(d, k, lanes=args.lanes), "batched_512": batched_512,
              "groupby_2e28": groupby_2e28, "groupby_wide": groupby_wide, "matmul_4096": matmul_4096, "fc_cfg1": fc_cfg1,
              "compressstore_masks": compressstore_masks, "sums_671m": sums_671m,
              "fc_1gib": lambda d, k: fc_1gib(d, max(3, min(k, 30)), 3)}[args.only]
        print(json.dumps({args.only: fn(dev, args.steps)}), flush=True)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
