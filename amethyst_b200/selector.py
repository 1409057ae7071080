"""Learned format and kernel-variant selector for operator chains, and the chain executors.

An operator chain is 2..5 operators drawn from {filter, compressstore, add, sub, mul, sum, min,
max, group-by-sum} applied to one packed column (semantics in chains.py).  Every operator that
produces a column (compressstore, add, sub, mul) is a *decision point* with up to six
candidates (chains.CANDIDATES): plain32, slabs at the natural width, slabs at the width rounded
to 8/16/32 bits, gap-free bits, slabs at the tightest width the value bound allows, and -- for a
binary op feeding a compressstore -- the fused kernel variant that runs both in one pass and
stores nothing in between.  The choice changes time, never values.  A small FP32 MLP
(amx_mlp_forward / amx_mlp_train_step, hand-written CUDA kernels) maps 16 features of a decision
point to a candidate.

Execution strategies:
  ChainRunner.program(choose)   the chain as one amx_program: device-resident lengths, no host
                                round trip, captured into a CUDA graph (alone, for timing, or with
                                other chains in one graph: ops.Graph)
  ChainRunner.run_plain()       the plain per-column, fixed-format form: one C-ABI call per
                                operator with every intermediate in slabs at its natural width,
                                and the survivor count read back to the host after each
                                compressstore to size the next call -- how the reference drives
                                its kernels (src/benchs/bench_compressstore_slabs.cu:60-62)

  sweep_labels(chain)  times every candidate of every decision point as a replayed CUDA graph of
                       the whole chain and labels it with the fastest -- the training data;
  exhaustive(chain)    times every combination of candidates: the yardstick for the selector's
                       regret and its fallback;
  Selector             the trained network.

The reference fixes every format at compile time (src/main.cu:300-340).  Nothing here changes the
integer arithmetic: the tests check that every strategy gives bit-identical results.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import torch

from . import _capi as A
from . import datagen, ops
from .chains import (BINARY_OPS, CANDIDATES, DECISION_OPS, DEFAULT_CHOICE, FUSED, K, MODEL_PATH, N_FEATURES, OPS,
                     ChainSpec, OpSpec, candidate_valid, decision_points, fixed, from_combo, key_bits, plan,
                     random_chain, valid_combos)

__all__ = ["ChainRunner", "Selector", "sweep_labels", "exhaustive", "evaluate", "train", "init_params", "OPS",
           "DECISION_OPS", "K", "CANDIDATES", "OpSpec", "ChainSpec", "random_chain", "FUSED", "time_graph"]


def time_graph(g: ops.Graph, reps: int = 5, stream=None) -> float:
    """Fastest of `reps` replays of a captured graph, in milliseconds (CUDA events on the
    launching stream), after one untimed replay."""
    s = stream if stream is not None else torch.cuda.current_stream()
    g.launch(s)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        g.launch(s)
        e1.record(s)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


class ChainRunner:
    """One chain's columns on the GPU: the input column, the right operands of its binary ops
    and the keys of its group-bys, the input's bit-width histogram, one result slot per
    operator (uint64; a compressstore's slot receives its survivor count) in `results`, and the
    group tables."""

    def __init__(self, chain: ChainSpec, results: torch.Tensor | None = None, slot0: int = 0, device="cuda"):
        self.chain = chain
        n = chain.n
        self.x0 = self._gen(n, chain.bits, chain.seed * 1009 + 1)
        self.aux = {}
        for i, op in enumerate(chain.ops):
            if op.kind in BINARY_OPS:
                self.aux[i] = self._gen(n, op.rhs_bits, chain.seed * 1009 + 17 + i)
            elif op.kind == "groupby":
                kb = key_bits(op.groups)
                cdf = np.arange(1, op.groups + 1, dtype=np.float64) / op.groups
                keys, _ = datagen.keys_from_cdf_gpu(n, cdf, chain.seed * 1009 + 33 + i)
                self.aux[i] = ops.convert(ops.PackedColumn(keys.view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, kb)
        self.hist = ops.bit_histogram(self.x0).cpu().numpy()
        self.results = results if results is not None else torch.zeros(len(chain.ops), dtype=torch.int64,
                                                                        device=device)
        self.slot0 = slot0
        self.groups = {}
        for i, op in enumerate(chain.ops):
            if op.kind == "groupby":
                g = 1 << self.aux[i].bits
                self.groups[i] = (ops.PackedColumn.empty(g, A.PLAIN32, 32), ops.PackedColumn.empty(g, A.PLAIN64, 64),
                                  ops.PackedColumn.empty(g, A.PLAIN64, 64))
        self._plain = None

    @staticmethod
    def _gen(n, bits, seed):
        plain = datagen.uniform_gpu(n, bits, seed)
        return ops.convert(ops.PackedColumn(plain.view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, bits)

    def slot_ptr(self, i: int) -> int:
        return self.results.data_ptr() + 8 * (self.slot0 + i)

    # ---------------------------------------------------------------- programs
    def program(self, choose) -> tuple:
        """(ops.Program, choices) for choose(i, feats, valid) -> candidate."""
        steps_plan, choices = plan(self.chain, choose, self.hist)
        steps = []
        for i, st in enumerate(steps_plan):
            s = A.Step()
            kind = st[0]
            if kind == "filter":
                s.kind = A.STEP_FILTER
                s.pred = ops.predicate(A.PRED_LT, st[1])
            elif kind == "compressstore":
                s.kind = A.STEP_COMPRESSSTORE
                s.pred = ops.predicate(A.PRED_LT, st[1])
                s.out_format, s.out_bits = st[2], st[3]
                s.d_result = self.slot_ptr(i)
            elif kind == "binary":
                s.kind = A.STEP_BINARY
                s.op, s.value_bits, s.out_format, s.out_bits = st[1], st[2], st[3], st[4]
                s.aux = self.aux[i].desc
            elif kind == "reduce":
                s.kind = A.STEP_REDUCE
                s.op = st[1]
                s.d_result = self.slot_ptr(i)
            else:
                s.kind = A.STEP_GROUPBY
                s.aux = self.aux[i].desc
                s.d_result = self.slot_ptr(i)
                gk, gs, gc = self.groups[i]
                s.group_keys, s.group_sums, s.group_counts = gk.desc, gs.desc, gc.desc
            steps.append(s)
        return ops.Program(self.x0, steps, keep=[self]), choices

    def time_program(self, prog: ops.Program, reps: int = 5) -> float:
        g = ops.Graph([prog], lanes=1)
        return time_graph(g, reps)

    def final_column(self, prog: ops.Program):
        """The final x of the program's last run (as a PackedColumn over its storage) and its
        length."""
        col, _ = prog.output()
        n = self._final_len()
        if col.data == self.x0.data.data_ptr():
            return ops.PackedColumn(self.x0.data, n, col.format, col.bits)
        off = col.data - prog.ws.data_ptr()
        return ops.PackedColumn(prog.ws[off:], n, col.format, col.bits)

    def _final_len(self) -> int:
        last = [i for i, o in enumerate(self.chain.ops) if o.kind == "compressstore"]
        if not last:
            return self.chain.n
        return int(self.results[self.slot0 + last[-1]].item())

    # ---------------------------------------------------------------- plain per-operator form
    def _plain_setup(self):
        """Buffers of the plain form: one output column per producing operator (capacity n,
        slabs at the natural width), one mask, one workspace, and the prepared descriptors."""
        ch = self.chain
        n = ch.n
        steps, _ = plan(ch, fixed(DEFAULT_CHOICE), self.hist)
        outs = {}
        for i, st in enumerate(steps):
            if st[0] == "compressstore":
                outs[i] = ops.PackedColumn.empty(n, st[2], st[3])
            elif st[0] == "binary":
                outs[i] = ops.PackedColumn.empty(n, st[3], st[4])
        mask = torch.zeros(ops.mask_words(n) + 4, dtype=torch.int32, device=self.x0.data.device)
        ws = ops.workspace(n)
        gws = {}
        for i in self.groups:
            t = ops.aligned_bytes(int(A.lib().amx_groupby_workspace_bytes(self.aux[i].bits)), 256)
            gws[i] = t
        preds = {i: ops.predicate(A.PRED_LT, st[1]) for i, st in enumerate(steps) if st[0] in ("filter", "compressstore")}
        self._plain = {"steps": steps, "outs": outs, "mask": mask, "ws": ws, "gws": gws, "preds": preds,
                       "host": torch.zeros(1, dtype=torch.int64, pin_memory=True)}

    def run_plain(self, stream=None):
        """The chain through the single-operator C ABI, slabs at the natural width everywhere;
        after each compressstore the survivor count comes back to the host (a synchronisation)
        so that the next call knows its length.  Results land in the same slots as a program's;
        returns the final column."""
        if self._plain is None:
            self._plain_setup()
        P = self._plain
        L = A.lib()
        s = C.c_void_p((stream if stream is not None else torch.cuda.current_stream()).cuda_stream)
        ws, wsb = C.c_void_p(P["ws"].data_ptr()), P["ws"].numel()
        maskp = C.c_void_p(P["mask"].data_ptr())
        x = self.x0
        n = self.chain.n
        xd = A.Column(x.data.data_ptr(), n, x.fmt, x.bits)
        live = False
        for i, st in enumerate(P["steps"]):
            kind = st[0]
            if kind == "filter":
                A.check(L.amx_filter(C.byref(xd), C.byref(P["preds"][i]), maskp, ws, wsb, s))
                live = True
            elif kind == "compressstore":
                o = P["outs"][i]
                od = A.Column(o.data.data_ptr(), n, o.fmt, o.bits)
                cnt = C.c_void_p(self.slot_ptr(i))
                if live:
                    A.check(L.amx_compressstore(C.byref(xd), maskp, C.byref(od), cnt, ws, wsb, s))
                else:
                    A.check(L.amx_filter_compressstore(C.byref(xd), C.byref(P["preds"][i]), C.byref(od), cnt, ws, wsb,
                                                       s))
                h = P["host"]
                h.copy_(self.results[self.slot0 + i: self.slot0 + i + 1], non_blocking=True)
                torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
                n = int(h[0])
                xd = A.Column(o.data.data_ptr(), n, o.fmt, o.bits)
                live = False
            elif kind == "binary":
                o = P["outs"][i]
                y = self.aux[i]
                yd = A.Column(y.data.data_ptr(), n, y.fmt, y.bits)
                od = A.Column(o.data.data_ptr(), n, o.fmt, o.bits)
                A.check(L.amx_binary(st[1], C.byref(xd), C.byref(yd), C.byref(od), ws, wsb, s))
                xd = od
            elif kind == "reduce":
                A.check(L.amx_reduce(st[1], C.byref(xd), maskp if live else None, C.c_void_p(self.slot_ptr(i)), ws,
                                     wsb, s))
            else:
                k = self.aux[i]
                kd = A.Column(k.data.data_ptr(), n, k.fmt, k.bits)
                gk, gs, gc = self.groups[i]
                g = P["gws"][i]
                A.check(L.amx_groupby(C.byref(kd), C.byref(xd), maskp if live else None, C.byref(gk.desc),
                                      C.byref(gs.desc), C.byref(gc.desc), C.c_void_p(self.slot_ptr(i)),
                                      C.c_void_p(g.data_ptr()), g.numel(), s))
        return xd

    def plain_final_column(self, xd: A.Column):
        if xd.data == self.x0.data.data_ptr():
            return ops.PackedColumn(self.x0.data, xd.n, xd.format, xd.bits)
        for o in self._plain["outs"].values():
            if o.data.data_ptr() == xd.data:
                return ops.PackedColumn(o.data, xd.n, xd.format, xd.bits)
        raise RuntimeError("unknown final column")

    # ---------------------------------------------------------------- digests
    def digest(self, final: ops.PackedColumn) -> list:
        """Host copies of a run's results for bit-exact comparison across strategies: every
        result slot (aggregates, survivor counts, group counts), every group table, and the
        final column's values decoded to uint64."""
        torch.cuda.synchronize()
        res = self.results[self.slot0: self.slot0 + len(self.chain.ops)].cpu().numpy().view(np.uint64).tolist()
        out = [("r", res)]
        for i in sorted(self.groups):
            g = int(res[i])
            gk, gs, gc = self.groups[i]
            out.append(("g", i, g, gk.data[: 4 * g].cpu().numpy().tobytes(), gs.data[: 8 * g].cpu().numpy().tobytes(),
                        gc.data[: 8 * g].cpu().numpy().tobytes()))
        if final.n:
            vals = ops.convert(final, A.PLAIN64, 64)
            out.append(("c", final.n, vals.host_bytes()))
        else:
            out.append(("c", 0))
        return out

    def clear_results(self):
        self.results[self.slot0: self.slot0 + len(self.chain.ops)].zero_()

    def decision_features(self) -> np.ndarray:
        """[decision points][16] features (they do not depend on the choices made)."""
        feats = []
        plan(self.chain, lambda i, f, valid: (feats.append(f), DEFAULT_CHOICE)[1], self.hist)
        return np.array(feats, np.float32).reshape(-1, N_FEATURES)

    def program_digest(self, choose) -> list:
        prog, _ = self.program(choose)
        self.clear_results()
        prog.run()
        return self.digest(self.final_column(prog))


def sweep_labels(chain: ChainSpec, reps: int = 3, runner: ChainRunner | None = None):
    """(features [d][16], labels [d], candidate times [d][K] with inf for candidates that do not
    exist there) for the chain's decision points.  Decision points are swept in order: each
    candidate is timed as the whole chain (replayed CUDA graph) with the earlier points at their
    fastest candidate and the later ones at the default."""
    runner = runner or ChainRunner(chain)
    feats = runner.decision_features()
    dps = decision_points(chain)
    chosen = []
    labels, times = [], []
    for j, i in enumerate(dps):
        t = np.full(K, np.inf)
        for c in range(K):
            combo = chosen + [c] + [DEFAULT_CHOICE] * (len(dps) - j - 1)
            if not candidate_valid(chain, i, c):
                continue
            prog, _ = runner.program(from_combo(combo))
            t[c] = runner.time_program(prog, reps)
        c = int(np.argmin(t))
        chosen.append(c)
        labels.append(c)
        times.append(t)
    return feats, np.array(labels, np.uint32), np.array(times).reshape(-1, K)


def exhaustive(chain: ChainSpec, runner: ChainRunner | None = None, reps: int = 3):
    """Times every valid combination of candidates as a replayed CUDA graph of the whole chain;
    returns (best ms, best combination, {combination: ms})."""
    runner = runner or ChainRunner(chain)
    table = {}
    for combo in valid_combos(chain):
        prog, _ = runner.program(from_combo(combo))
        table[combo] = runner.time_program(prog, reps)
    bc = min(table, key=table.get)
    return table[bc], bc, table


class Selector:
    """The trained network: parameters on the GPU, amx_mlp_forward for every decision."""

    def __init__(self, params: np.ndarray, confidence: float = 0.0, device="cuda"):
        self.params = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(device)
        self.confidence = confidence
        self.fallbacks = 0
        self.decisions = 0

    @staticmethod
    def load(path: str = MODEL_PATH, confidence: float = 0.0) -> "Selector":
        d = np.load(path)
        if int(d["classes"]) != K:
            raise ValueError(f"{path}: a model for {int(d['classes'])} candidates, {K} expected")
        return Selector(d["params"], confidence)

    def probs(self, feats: np.ndarray) -> np.ndarray:
        x = torch.from_numpy(np.ascontiguousarray(feats, np.float32).reshape(-1, N_FEATURES)).cuda()
        p = torch.empty(max(1, x.shape[0]), K, dtype=torch.float32, device="cuda")
        if x.shape[0]:
            A.check(A.lib().amx_mlp_forward(C.c_void_p(self.params.data_ptr()), K, C.c_void_p(x.data_ptr()),
                                            x.shape[0], C.c_void_p(p.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return p[: x.shape[0]].cpu().numpy()

    def decide_fn(self, runner: ChainRunner | None = None):
        """choose(i, feats, valid) for ChainRunner.program: the network's most probable valid
        candidate, or -- below the confidence threshold and with a runner at hand -- the fastest
        candidate of that decision timed on the spot."""

        def choose(i, feats, valid):
            self.decisions += 1
            p = self.probs(feats)[0]
            c = max(valid, key=lambda k: p[k])
            if p[c] < self.confidence and runner is not None:
                self.fallbacks += 1
                best, bt = c, float("inf")
                for k in valid:
                    prog, _ = runner.program(lambda j, f, v, k=k: k if j == i else DEFAULT_CHOICE)
                    t = runner.time_program(prog, 2)
                    if t < bt:
                        best, bt = k, t
                c = best
            return c

        return choose

    def choices(self, runners: list) -> list:
        """The network's picks for every decision point of many chains in one forward pass."""
        feats = [r.decision_features() for r in runners]
        allf = np.concatenate([f for f in feats if len(f)] or [np.zeros((0, N_FEATURES), np.float32)])
        p = self.probs(allf) if len(allf) else np.zeros((0, K), np.float32)
        out, k = [], 0
        for r, f in zip(runners, feats):
            picks = []
            for i in decision_points(r.chain):
                valid = [c for c in range(K) if candidate_valid(r.chain, i, c)]
                picks.append(max(valid, key=lambda c: p[k][c]))
                k += 1
            out.append(tuple(picks))
            self.decisions += len(picks)
        return out


def init_params(seed: int = 1) -> np.ndarray:
    """He-uniform weights, zero biases, in the layout of amx_mlp_param_count(K)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in [(N_FEATURES, 64), (64, 64), (64, K)]:
        lim = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, size=fan_out * fan_in).astype(np.float32))
        parts.append(np.zeros(fan_out, np.float32))
    p = np.concatenate(parts)
    assert p.size == int(A.lib().amx_mlp_param_count(K))
    return p


def train(feats: np.ndarray, labels: np.ndarray, epochs=60, batch=256, lr=3e-3, seed=1):
    """Mini-batch Adam on the GPU (amx_mlp_train_step).  Returns (params, per-epoch mean loss)."""
    L = A.lib()
    p = torch.from_numpy(init_params(seed)).cuda()
    adam = torch.zeros(2 * p.numel(), dtype=torch.float32, device="cuda")
    x = torch.from_numpy(np.ascontiguousarray(feats, np.float32)).cuda()
    y = torch.from_numpy(np.ascontiguousarray(labels, np.uint32).view(np.int32)).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(seed)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    step, hist = 0, []
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(len(labels))).cuda()
        xp, yp = x[perm].contiguous(), y[perm].contiguous()
        tot = 0.0
        for b0 in range(0, len(labels), batch):
            nb = min(batch, len(labels) - b0)
            step += 1
            A.check(L.amx_mlp_train_step(C.c_void_p(p.data_ptr()), C.c_void_p(adam.data_ptr()), step, K,
                                         C.c_void_p(xp[b0:].data_ptr()), C.c_void_p(yp[b0:].data_ptr()), nb,
                                         C.c_float(lr), C.c_void_p(loss.data_ptr()), s))
            tot += float(loss.item()) * nb
        hist.append(tot / max(1, len(labels)))
    return p.cpu().numpy(), hist


def evaluate(selector: Selector, chains, reps: int = 3, check_exact: bool = True):
    """Per held-out chain: the exhaustive best, the selector's pick and the fixed plain32 and
    fixed natural-slab strategies, each timed as a replayed CUDA graph of the whole chain; every
    strategy's results are checked bit-identical to the plain per-operator form's."""
    rows = []
    for ch in chains:
        runner = ChainRunner(ch)
        best_ms, best_combo, table = exhaustive(ch, runner, reps)
        runner.clear_results()
        xd = runner.run_plain()
        ref = runner.digest(runner.plain_final_column(xd)) if check_exact else None
        pick = selector.choices([runner])[0]
        row = {"ops": [o.kind for o in ch.ops], "n": ch.n, "bits": ch.bits, "best_ms": best_ms,
               "best": list(best_combo), "selector": list(pick), "combos": len(table)}
        for name, combo in [("selector", pick), ("plain32", tuple(0 for _ in best_combo)),
                            ("slab", tuple(DEFAULT_CHOICE for _ in best_combo)), ("best", best_combo)]:
            row[name + "_ms"] = table[combo]
            if check_exact:
                row[name + "_exact"] = runner.program_digest(from_combo(combo)) == ref
        rows.append(row)
        del runner
        torch.cuda.empty_cache()
    sel = np.array([r["selector_ms"] for r in rows])
    best = np.array([r["best_ms"] for r in rows])
    regret = sel / best - 1.0
    summary = {
        "chains": len(rows),
        "median_regret": float(np.median(regret)), "mean_regret": float(np.mean(regret)),
        "p90_regret": float(np.percentile(regret, 90)),
        "total_ms": {"exhaustive_best": float(best.sum()), "selector": float(sel.sum()),
                     "plain32": float(sum(r["plain32_ms"] for r in rows)),
                     "slab": float(sum(r["slab_ms"] for r in rows))},
        "speedup_vs_plain32": float(sum(r["plain32_ms"] for r in rows) / sel.sum()),
        "speedup_vs_slab": float(sum(r["slab_ms"] for r in rows) / sel.sum()),
        "all_exact": all(r.get(k + "_exact", True) for r in rows for k in ("selector", "plain32", "slab", "best")),
        "decisions": selector.decisions,
    }
    return summary, rows


def main(argv=None):
    """Sweep `--train` synthetic chains for labels, train the network, evaluate it on `--eval`
    held-out chains against the exhaustive best, and write the model and a JSON report."""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--eval", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=80)
    ap.add_argument("--model", default=MODEL_PATH)
    ap.add_argument("--report", default="selector_report.json")
    ap.add_argument("--data", default=None, help="reuse a saved sweep (npz) instead of sweeping")
    args = ap.parse_args(argv)
    t0 = time.time()
    if args.data and os.path.exists(args.data):
        d = np.load(args.data)
        feats, labels, times = d["feats"], d["labels"], d["times"]
    else:
        rng = np.random.default_rng(2024)
        fs, ls, ts = [], [], []
        for k in range(args.train):
            ch = random_chain(rng, seed=k + 1)
            if not decision_points(ch):
                continue
            f, l, t = sweep_labels(ch, reps=3)
            fs.append(f)
            ls.append(l)
            ts.append(t)
            if k % 256 == 0:
                torch.cuda.empty_cache()
        feats, labels, times = np.concatenate(fs), np.concatenate(ls), np.concatenate(ts)
        if args.data:
            np.savez_compressed(args.data, feats=feats, labels=labels, times=times)
    t_sweep = time.time() - t0
    # 90 / 10 split of the decision points for a validation accuracy
    idx = np.random.default_rng(7).permutation(len(labels))
    cut = int(0.9 * len(idx))
    tr, va = idx[:cut], idx[cut:]
    params, hist = train(feats[tr], labels[tr], epochs=args.epochs)
    sel = Selector(params)
    pv = sel.probs(feats[va]) if len(va) else np.zeros((0, K))
    tv = times[va]
    pv = np.where(np.isfinite(tv), pv, -1.0).argmax(1) if len(va) else np.array([], int)
    acc = float((pv == labels[va]).mean()) if len(va) else float("nan")
    dec_regret = (tv[np.arange(len(va)), pv] / tv.min(1) - 1.0) if len(va) else np.array([0.0])
    params, hist = train(feats, labels, epochs=args.epochs)  # final model on every point
    np.savez(args.model, params=params, classes=K, features=N_FEATURES,
             label_hist=np.bincount(labels, minlength=K))
    sel = Selector(params)
    t1 = time.time()
    rng = np.random.default_rng(99)
    held = [random_chain(rng, seed=100000 + k) for k in range(args.eval)]
    held = [c for c in held if decision_points(c)]
    summary, rows = evaluate(sel, held)
    report = {"train_chains": args.train, "decision_points": int(len(labels)),
              "label_histogram": np.bincount(labels, minlength=K).tolist(),
              "candidates": [f"{A.FORMAT_NAMES.get(f, 'fused')}/{w}" for f, w in CANDIDATES],
              "loss_first_last": [hist[0], hist[-1]], "validation_accuracy": acc,
              "validation_decision_regret_median": float(np.median(dec_regret)),
              "sweep_seconds": t_sweep, "eval_seconds": time.time() - t1, "eval": summary}
    with open(args.report, "w") as f:
        json.dump({"report": report, "rows": rows}, f, indent=1, default=str)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
