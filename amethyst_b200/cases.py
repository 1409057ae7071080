"""Named single-GPU workloads of the operator layer, for timing and profiling one kernel at a time.

    python -m amethyst_b200.cases <case> [reps]

prints one JSON line with the mean milliseconds per call (CUDA events, after 3 warm-up calls) and
packed GB/s (or TOPS for the matrix multiply).  Inputs are generated on the GPU (seeded) and are
larger than the 126 MB L2 unless the case says otherwise.

  chain      A 2^26 x u7 slabs + B 2^26 x u13 slabs -> C at 14 bits, keep C >= 2^13, compressstore
             to 14-bit slabs, sum (one amx_chain call)
  fcB        filter v < 205 * 2^(B-11) + compressstore over 2^24 slabs of width B (e.g. fc11)
  fc_cfg1    filter v < 205 + compressstore over 2^24 elements in 11-bit slabs (26.8 MB)
  filterB    filter -> bitmask over 2^24 slabs of width B
  sumB       sum of every value of 2^24 slabs of width B (amx_reduce: no predicate, no mask)
  matmul     4096^3 u7 x u7 slab matrices -> narrowest-width slabs (unpack + GEMM + pack)
  matmul_fused  the same through the fused kernel (amx_tuning.policy 2)
  batch64    64 slab columns, lengths log-uniform in [2^16, 2^22], widths 1..32: one batch run
  groupby    2^26 Zipf(1.1) keys over 1000 groups at 10 bits, 2^26 u16 values at 16 bits
  groupby32  2^26 Zipf(1.1) keys drawn from 100,000 random 32-bit keys (32-bit slabs), 2^26 u16
             values: the wide-key hash table, the 512 MB key bitmap and the ordered extraction
  groupby32_sort  the same through the sort-based group-by (radix sort + reduce-by-key)
  mixed64    the 64 held-out operator chains of the mixed-chain bench line as one CUDA graph of
             selector-planned programs (8 lanes); each timed replay runs inside the NVTX range
             "mixed64-replay", so a profiler can list that replay's kernels alone
"""
from __future__ import annotations

import ctypes as C
import json
import sys

import numpy as np
import torch

from . import _capi as A
from . import datagen, ops


def _gen(n, bits, seed, fmt=A.SLAB):
    plain = datagen.uniform_gpu(n, bits, seed)
    return ops.convert(ops.PackedColumn(plain.view(torch.uint8), n, A.PLAIN32, 32), fmt, bits)


def _time(fn, reps):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def case(name: str, reps: int = 10) -> dict:
    L = A.lib()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if name == "chain":
        n = 1 << 26
        a, b = _gen(n, 7, 0x5EEDA), _gen(n, 13, 0x5EEDB)
        out = ops.PackedColumn.empty(n, A.SLAB, 14)
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        agg = torch.zeros(2, dtype=torch.int64, device="cuda")
        ws = ops.workspace(n)
        desc = A.ChainDesc(A.OP_ADD, 14, ops.predicate(A.PRED_GE, 1 << 13, 0, 14), A.AGG_SUM, 0)
        ad, bd, od = a.desc, b.desc, out.desc

        def step():
            A.check(L.amx_chain(C.byref(desc), C.byref(ad), C.byref(bd), C.byref(od), None,
                                C.c_void_p(cnt.data_ptr()), C.c_void_p(agg.data_ptr()), C.c_void_p(ws.data_ptr()),
                                ws.numel(), s))

        ms = _time(step, reps)
        byts = a.nbytes + b.nbytes + ops.storage_bytes(A.SLAB, 14, int(cnt[0].item())) + 16
        return {"case": name, "ms": ms, "GB_s": byts / ms / 1e6}
    if name.startswith("sum"):
        bits = int(name[3:])
        n = (1 << 24) * (64 // bits)
        col = _gen(n, bits, 0xC0FFEE)
        ws = ops.workspace(n)
        res = torch.zeros(2, dtype=torch.int64, device="cuda")
        cd = col.desc

        def step():
            A.check(L.amx_reduce(A.AGG_SUM, C.byref(cd), None, C.c_void_p(res.data_ptr()), C.c_void_p(ws.data_ptr()),
                                 ws.numel(), s))

        ms = _time(step, reps)
        return {"case": name, "ms": ms, "GB_s": (col.nbytes + 8) / ms / 1e6}
    if name.startswith("fc") or name.startswith("filter"):
        flt = name.startswith("filter")
        small = name == "fc_cfg1"  # the plain configuration: 2^24 elements (not slabs) at 11 bits
        bits = 11 if small else int(name[6:] if flt else name[2:])
        n = (1 << 24) if small else (1 << 24) * (64 // bits)
        col = _gen(n, bits, 0xC0FFEE)
        ws = ops.workspace(n)
        thr = (205 << (bits - 11)) if bits >= 11 else max(1, 205 >> (11 - bits))
        pred = ops.predicate(A.PRED_LT, thr, 0, bits)
        cd = col.desc
        if flt:
            mask = torch.zeros(n // 32 + 64, dtype=torch.int32, device="cuda")

            def step():
                A.check(L.amx_filter(C.byref(cd), C.byref(pred), C.c_void_p(mask.data_ptr()),
                                     C.c_void_p(ws.data_ptr()), ws.numel(), s))

            ms = _time(step, reps)
            return {"case": name, "ms": ms, "GB_s": (col.nbytes + n // 8) / ms / 1e6}
        out = ops.PackedColumn.empty(n, A.SLAB, bits)
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        od = out.desc

        def step():
            A.check(L.amx_filter_compressstore(C.byref(cd), C.byref(pred), C.byref(od), C.c_void_p(cnt.data_ptr()),
                                               C.c_void_p(ws.data_ptr()), ws.numel(), s))

        ms = _time(step, reps)
        byts = col.nbytes + ops.storage_bytes(A.SLAB, bits, int(cnt[0].item())) + 8
        return {"case": name, "ms": ms, "GB_s": byts / ms / 1e6}
    if name in ("matmul", "matmul_fused"):
        M = N = K = 4096
        if name == "matmul_fused":
            A.check(L.amx_set_tuning(C.byref(A.Tuning(0, 0, 2, 0))))

        def slab_matrix(rows, cols, bits, seed):
            eps = 64 // bits
            rs = (cols + eps - 1) // eps
            plain = datagen.uniform_gpu(rows * cols, bits, seed).view(rows, cols)
            pad = torch.zeros(rows, rs * eps, dtype=torch.int32, device="cuda")
            pad[:, :cols] = plain
            flat = ops.PackedColumn(pad.reshape(-1).contiguous().view(torch.uint8), rows * rs * eps, A.PLAIN32, 32)
            c = ops.convert(flat, A.SLAB, bits)
            return ops.PackedColumn(c.data, rows * cols, A.SLAB, bits)

        a, b = slab_matrix(M, K, 7, 0xA11), slab_matrix(K, N, 7, 0xB22)
        ws = ops.matmul_workspace(M, N, K)
        out, width = ops.matmul(a, b, M, N, K, ws=ws)

        def step():
            A.check(L.amx_matmul(C.byref(a.desc), C.byref(b.desc), M, N, K, C.byref(out.desc),
                                 C.c_void_p(width.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(), s))

        ms = _time(step, reps)
        return {"case": name, "ms": ms, "TOPS": 2 * M * N * K / ms / 1e9, "out_bits": int(width[0].item())}
    if name == "batch64":
        rng = np.random.default_rng(5)
        cols, preds = [], []
        for i in range(64):
            n = int(np.exp(rng.uniform(np.log(2 ** 16), np.log(2 ** 22))))
            w = int(rng.integers(1, 33))
            cols.append(_gen(n, w, 77 + i))
            preds.append(ops.predicate(A.PRED_LT, max(1, int(rng.uniform(0.01, 0.99) * (1 << w))), 0, w))
        b = ops.Batch(cols, preds, A.BatchTuning(512, 2))
        ms = _time(b.run, reps)
        tot = sum(ops.storage_bytes(A.SLAB, c.bits, c.n) for c in cols)
        return {"case": name, "ms": ms, "GB_s": tot / ms / 1e6}
    if name == "groupby":
        n = 1 << 26
        k32, _ = datagen.keys_from_cdf_gpu(n, datagen.zipf_cdf(1000, 1.1), 3)
        keys = ops.convert(ops.PackedColumn(k32.view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, 10)
        vals = _gen(n, 16, 4)
        gws = torch.empty(int(L.amx_groupby_workspace_bytes(10)) + 256, dtype=torch.uint8, device="cuda")
        gws = gws[(-gws.data_ptr()) % 256:]
        ms = _time(lambda: ops.groupby(keys, vals, ws=gws), reps)
        return {"case": name, "ms": ms, "GB_s": (keys.nbytes + vals.nbytes) / ms / 1e6}
    if name in ("groupby32", "groupby32_sort"):
        n, groups = 1 << 26, 100000
        idx, _ = datagen.keys_from_cdf_gpu(n, datagen.zipf_cdf(groups, 1.1), 5)
        pool = torch.from_numpy(np.random.default_rng(6).choice(1 << 32, size=groups, replace=False)).cuda()
        k32 = pool[idx[:n].long()].to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.int32)
        keys = ops.convert(ops.PackedColumn(k32.contiguous().view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, 32)
        vals = _gen(n, 16, 7)
        if name == "groupby32_sort":
            sws = ops.aligned_bytes(int(L.amx_groupby_sort_workspace_bytes(n, 32, 16)), 256)
            ms = _time(lambda: ops.groupby_sort(keys, vals, ws=sws, max_groups=1 << 17), reps)
            A.check(L.amx_groupby_sort_status(C.c_void_p(sws.data_ptr()), s))
        else:
            gws = ops.groupby_workspace(32, 1 << 17)
            ms = _time(lambda: ops.groupby(keys, vals, ws=gws, max_groups=1 << 17), reps)
            ops.groupby_status(gws, 32)
        return {"case": name, "ms": ms, "GB_s": (keys.nbytes + vals.nbytes) / ms / 1e6}
    if name == "mixed64":
        from . import chains as X
        from . import selector as S

        rng = np.random.default_rng(99)
        specs, k = [], 0
        while len(specs) < 64:
            ch = X.random_chain(rng, seed=100000 + k)
            k += 1
            if X.decision_points(ch):
                specs.append(ch)
        results = torch.zeros(sum(len(c.ops) for c in specs), dtype=torch.int64, device="cuda")
        runners, slot = [], 0
        for ch in specs:
            runners.append(S.ChainRunner(ch, results, slot))
            slot += len(ch.ops)
        picks = S.Selector.load().choices(runners)
        progs = [r.program(X.from_combo(p))[0] for r, p in zip(runners, picks)]
        g = ops.Graph(progs, lanes=8)

        def replay():
            torch.cuda.nvtx.range_push("mixed64-replay")
            g.launch()
            torch.cuda.nvtx.range_pop()

        ms = _time(replay, reps)
        return {"case": name, "ms": ms, "elements": int(sum(c.n for c in specs))}
    raise ValueError(f"unknown case {name}")


if __name__ == "__main__":
    print(json.dumps(case(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 10)))
