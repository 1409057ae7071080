"""Learned format selector for operator chains.

An operator chain is 2..5 operators drawn from {filter, compressstore, add, sub, mul, sum, min,
max, group-by-sum} applied to one packed column.  Every operator that produces a column
(compressstore, add, sub, mul) is a *decision point*: its output can be stored as
  0  plain32 at the natural width,
  1  slabs at the natural width,
  2  slabs at the width rounded up to 8 / 16 / 32 bits,
  3  the gap-free bit stream at the natural width,
and the choice changes the time of the operator and of the operator that reads its output, never
the values.  A small FP32 MLP (amx_mlp_forward / amx_mlp_train_step, hand-written CUDA kernels)
maps 16 features of the decision point to one of the four candidates.

  sweep_labels(chain)  times every candidate of every decision point (the operator plus its
                       consumer, CUDA events) and labels it with the fastest -- the training data;
  exhaustive(chain)    times every combination of candidates for a whole chain: the yardstick for the
                       selector's regret and its fallback;
  Selector             the trained network; `decide` falls back to timing the candidates on the
                       spot when its top probability is below `confidence`.

The reference picks formats at compile time for each benchmark (src/main.cu:300-340); nothing
here changes the integer arithmetic, and the tests check that every strategy gives bit-identical
results.
"""
from __future__ import annotations

import ctypes as C
import itertools
import math
import os

import numpy as np
import torch

from . import _capi as A
from . import datagen, ops

from .chains import (CANDIDATES, DECISION_OPS, DEFAULT_CHOICE, K, MODEL_PATH, N_FEATURES, OPS, ChainSpec, OpSpec,
                     candidate_bits, features, natural_out_bits, random_chain)

class ChainRunner:
    """Holds one chain's input and auxiliary columns on the GPU and executes it under any choice
    of candidates, timing every operator with CUDA events."""

    AGG = {"sum": A.AGG_SUM, "min": A.AGG_MIN, "max": A.AGG_MAX}
    BIN = {"add": A.OP_ADD, "sub": A.OP_SUB, "mul": A.OP_MUL}

    def __init__(self, chain: ChainSpec, device="cuda"):
        self.chain = chain
        self.x0 = self._gen(chain.n, chain.bits, chain.seed * 1009 + 1)
        self.aux = {}
        for i, op in enumerate(chain.ops):
            if op.kind in self.BIN:
                self.aux[i] = self._gen(chain.n, op.rhs_bits, chain.seed * 1009 + 17 + i)
            elif op.kind == "groupby":
                kb = max(1, (op.groups - 1).bit_length())
                cdf = np.arange(1, op.groups + 1, dtype=np.float64) / op.groups
                keys, _ = datagen.keys_from_cdf_gpu(chain.n, cdf, chain.seed * 1009 + 33 + i)
                self.aux[i] = ops.convert(ops.PackedColumn(keys.view(torch.uint8), chain.n, A.PLAIN32, 32), A.SLAB, kb)
        self.ws = ops.workspace(chain.n)
        self.gws = {i: torch.empty(int(A.lib().amx_groupby_workspace_bytes(self.aux[i].bits)) + 256,
                                   dtype=torch.uint8, device=device)
                    for i, op in enumerate(chain.ops) if op.kind == "groupby"}
        for i in self.gws:
            t = self.gws[i]
            off = (-t.data_ptr()) % 256
            self.gws[i] = t[off:]

    @staticmethod
    def _gen(n, bits, seed):
        plain = datagen.uniform_gpu(n, bits, seed)
        return ops.convert(ops.PackedColumn(plain.view(torch.uint8), n, A.PLAIN32, 32), A.SLAB, bits)

    @staticmethod
    def _prefix(col, n):
        return ops.PackedColumn(col.data, n, col.fmt, col.bits)

    def _pred(self, sel, w):
        return ops.predicate(A.PRED_LT, max(1, int(round(sel * (1 << w)))), 0, w)

    def run_op(self, i, state, choice):
        """Executes operator i on state (x, mask, w) -- w is the natural width of x's values,
        which may be stored wider -- with candidate `choice` for its output; returns (new state,
        result or None, milliseconds)."""
        x, mask, w = state
        op = self.chain.ops[i]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        result = None
        e0.record()
        if op.kind == "filter":
            mask = ops.filter(x, self._pred(op.sel, w), ws=self.ws)
        elif op.kind == "compressstore":
            fmt, _ = CANDIDATES[choice]
            sw = candidate_bits(choice, w)
            if mask is not None:
                out, cnt = ops.compressstore(x, mask, fmt, sw, ws=self.ws)
            else:
                out, cnt = ops.filter_compressstore(x, self._pred(op.sel, w), fmt, sw, ws=self.ws)
            e1.record()
            e1.synchronize()
            n2 = int(cnt[0].item())
            return (ops.PackedColumn(out.data, n2, fmt, sw), None, w), None, e0.elapsed_time(e1)
        elif op.kind in self.BIN:
            y = self._prefix(self.aux[i], x.n)
            ow = natural_out_bits(op.kind, w, y.bits)
            fmt, _ = CANDIDATES[choice]
            x = ops.binary_op(self.BIN[op.kind], x, y, fmt, candidate_bits(choice, ow, op.kind), ws=self.ws)
            w = ow
        elif op.kind in self.AGG:
            result = ops.hop(self.AGG[op.kind], x, mask, ws=self.ws)
        else:  # group-by-sum of the column's values by the auxiliary keys
            keys = self._prefix(self.aux[i], x.n)
            result = ops.groupby(keys, x, mask=mask, ws=self.gws[i])
        e1.record()
        e1.synchronize()
        return (x, mask, w), result, e0.elapsed_time(e1)

    def decision_features(self, i, state):
        x, _, w = state
        op = self.chain.ops[i]
        ow = natural_out_bits(op.kind, w, self.aux[i].bits) if op.kind in self.BIN else w
        return features(self.chain, i, x.n, w, ow)

    def run(self, choose):
        """Whole chain; choose(i, feats, state) -> candidate for decision point i.  Returns
        (total milliseconds, results, final column, choices)."""
        state = (self.x0, None, self.chain.bits)
        total, results, choices = 0.0, [], []
        for i, op in enumerate(self.chain.ops):
            c = DEFAULT_CHOICE
            if op.kind in DECISION_OPS:
                c = choose(i, self.decision_features(i, state), state)
                choices.append(c)
            state, res, ms = self.run_op(i, state, c)
            total += ms
            if res is not None:
                results.append(res)
        return total, results, state[0], choices

    def digest(self, results, final) -> list:
        """Host copies of a run's results for bit-exact comparison across strategies: every
        aggregate, every group table, and the final column's values decoded to uint64."""
        out = []
        for r in results:
            if isinstance(r, tuple):
                ok, osum, ocnt, ng = r
                g = int(ng[0].item())
                vals = ops.convert(ops.PackedColumn(ok.data, g, ok.fmt, ok.bits), A.PLAIN64, 64)
                out.append(("g", g, vals.host_bytes(), osum.data[: 8 * g].cpu().numpy().tobytes(),
                            ocnt.data[: 8 * g].cpu().numpy().tobytes()))
            else:
                out.append(("a", int(r.cpu().numpy().view(np.uint64)[0])))
        if final.n:
            vals = ops.convert(final, A.PLAIN64, 64)
            out.append(("c", final.n, vals.host_bytes()))
        else:
            out.append(("c", 0))
        return out


def _time_candidate(runner, i, state, c, reps=3):
    """Operator i with candidate c plus the operator that reads its output (default choice)."""
    best = float("inf")
    for r in range(reps + 1):
        s2, _, ms = runner.run_op(i, state, c)
        if i + 1 < len(runner.chain.ops):
            _, _, ms2 = runner.run_op(i + 1, s2, DEFAULT_CHOICE)
            ms += ms2
        if r:  # the first run warms up
            best = min(best, ms)
    return best


def sweep_labels(chain: ChainSpec, reps=3):
    """(features [d][16], labels [d], candidate times [d][K]) for the chain's decision points;
    the chain proceeds along the fastest candidate of each point."""
    runner = ChainRunner(chain)
    feats, labels, times = [], [], []
    state = (runner.x0, None, chain.bits)
    for i, op in enumerate(chain.ops):
        c = DEFAULT_CHOICE
        if op.kind in DECISION_OPS:
            t = [_time_candidate(runner, i, state, k, reps) for k in range(K)]
            c = int(np.argmin(t))
            feats.append(runner.decision_features(i, state))
            labels.append(c)
            times.append(t)
        state, _, _ = runner.run_op(i, state, c)
    return (np.array(feats, np.float32).reshape(-1, N_FEATURES), np.array(labels, np.uint32),
            np.array(times).reshape(-1, K))


def exhaustive(chain: ChainSpec, runner: ChainRunner | None = None, reps=2):
    """Times every combination of candidates; returns (best ms, best combination, {combo: ms})."""
    runner = runner or ChainRunner(chain)
    d = sum(1 for o in chain.ops if o.kind in DECISION_OPS)
    table = {}
    for combo in itertools.product(range(K), repeat=d):
        best = float("inf")
        for r in range((reps if d <= 3 else 1) + 1):
            it = iter(combo)
            ms, _, _, _ = runner.run(lambda i, f, st: next(it))
            if r:
                best = min(best, ms)
        table[combo] = best
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
        return Selector(np.load(path)["params"], confidence)

    def probs(self, feats: np.ndarray) -> np.ndarray:
        x = torch.from_numpy(np.ascontiguousarray(feats, np.float32).reshape(-1, N_FEATURES)).cuda()
        p = torch.empty(x.shape[0], K, dtype=torch.float32, device="cuda")
        A.check(A.lib().amx_mlp_forward(C.c_void_p(self.params.data_ptr()), K, C.c_void_p(x.data_ptr()), x.shape[0],
                                        C.c_void_p(p.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return p.cpu().numpy()

    def decide_fn(self, runner: ChainRunner | None = None):
        """choose(i, feats, state) for ChainRunner.run: the network's pick, or -- below the
        confidence threshold and with a runner at hand -- the fastest candidate timed on the spot
        (the exhaustive sweep of that one decision)."""

        def choose(i, feats, state):
            self.decisions += 1
            p = self.probs(feats)[0]
            c = int(np.argmax(p))
            if p[c] < self.confidence and runner is not None:
                self.fallbacks += 1
                t = [_time_candidate(runner, i, state, k, 1) for k in range(K)]
                c = int(np.argmin(t))
            return c

        return choose


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


def evaluate(selector: Selector, chains, exhaustive_reps=2):
    """Per held-out chain: the exhaustive best, the selector's pick, and the fixed plain32 and
    fixed natural-slab strategies, each timed end to end (sum of the operators' CUDA-event times);
    every strategy's results are checked bit-identical to the exhaustive best's."""
    rows = []
    for ch in chains:
        runner = ChainRunner(ch)
        best_ms, best_combo, _ = exhaustive(ch, runner, exhaustive_reps)
        it = iter(best_combo)
        _, r_best, f_best, _ = runner.run(lambda i, f, st: next(it))
        ref = runner.digest(r_best, f_best)
        row = {"ops": [o.kind for o in ch.ops], "n": ch.n, "bits": ch.bits, "best_ms": best_ms,
               "best": list(best_combo)}
        for name, choose in [("selector", selector.decide_fn(runner)),
                             ("plain32", lambda i, f, st: 0), ("slab", lambda i, f, st: 1)]:
            runner.run(choose)  # warm-up
            t = []
            for _ in range(exhaustive_reps):
                ms, res, fin, picks = runner.run(choose)
                t.append(ms)
            row[name + "_ms"] = min(t)
            row[name + "_picks"] = picks
            row[name + "_exact"] = runner.digest(res, fin) == ref
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
        "all_exact": all(r["selector_exact"] and r["plain32_exact"] and r["slab_exact"] for r in rows),
        "fallbacks": selector.fallbacks, "decisions": selector.decisions,
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
            f, l, t = sweep_labels(random_chain(rng, seed=k + 1), reps=2)
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
    pv = sel.probs(feats[va]).argmax(1) if len(va) else np.array([])
    acc = float((pv == labels[va]).mean()) if len(va) else float("nan")
    # per-decision regret of the network's pick on the validation points (candidate times known)
    dec_regret = (times[va][np.arange(len(va)), pv] / times[va].min(1) - 1.0) if len(va) else np.array([0.0])
    params, hist = train(feats, labels, epochs=args.epochs)  # final model on every point
    np.savez(args.model, params=params, classes=K, features=N_FEATURES,
             label_hist=np.bincount(labels, minlength=K))
    sel = Selector(params)
    t1 = time.time()
    rng = np.random.default_rng(99)
    held = [random_chain(rng, seed=100000 + k) for k in range(args.eval)]
    summary, rows = evaluate(sel, held)
    report = {"train_chains": args.train, "decision_points": int(len(labels)),
              "label_histogram": np.bincount(labels, minlength=K).tolist(),
              "candidates": [f"{A.FORMAT_NAMES[f]}/{w}" for f, w in CANDIDATES],
              "loss_first_last": [hist[0], hist[-1]], "validation_accuracy": acc,
              "validation_decision_regret_median": float(np.median(dec_regret)),
              "sweep_seconds": t_sweep, "eval_seconds": time.time() - t1, "eval": summary}
    with open(args.report, "w") as f:
        json.dump({"report": report, "rows": rows}, f, indent=1, default=str)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
