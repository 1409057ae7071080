"""Operator chains for the format selector: the synthetic chain distribution, the candidates of a
decision point, value-bound tracking, the 16 features the selector network reads, and the
translation of a chain plus one candidate per decision point into the steps of an amx_program.
Host logic only (no torch, no GPU), shared by the selector, the benchmark and their CPU tests.

Chain semantics (the same for every execution strategy, so all of them give identical results):
the state is a column x of n elements with a semantic value width w, plus an optional live mask.
  filter         mask = (x < k), k = max(1, round(sel * 2^w))
  compressstore  x = x[mask] (x[x < k] without a live mask); the mask is consumed
  add/sub/mul    x = op(x, y[0..len)) masked to the natural width (add: max+1, mul: sum of the
                 widths, sub: max, all capped at 32 bits); y is an auxiliary column of rhs_bits
  sum/min/max    one uint64 aggregate of x (of the masked elements when a mask is live)
  groupby        group-by sum + count of x by an auxiliary key column (masked)
The reference chains operators one launch at a time (src/op_chaining_demo.cu:137-152).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from ._capi import (AGG_MAX, AGG_MIN, AGG_SUM, FORMAT_FUSED, NOGAPS, OP_ADD, OP_MUL, OP_SUB, PLAIN32, SLAB,
                    STEP_BINARY, STEP_COMPRESSSTORE, STEP_FILTER, STEP_GROUPBY, STEP_REDUCE)

OPS = ["filter", "compressstore", "add", "sub", "mul", "sum", "min", "max", "groupby"]
DECISION_OPS = {"compressstore", "add", "sub", "mul"}
BINARY_OPS = {"add": OP_ADD, "sub": OP_SUB, "mul": OP_MUL}
AGG_OPS = {"sum": AGG_SUM, "min": AGG_MIN, "max": AGG_MAX}
# what a decision point can do with the column it produces: a storage format and width rule, or
# (binary op before a compressstore) the fused kernel variant that never stores it
CANDIDATES = [(PLAIN32, "natural"), (SLAB, "natural"), (SLAB, "byte"), (NOGAPS, "natural"), (SLAB, "tight"),
              (FORMAT_FUSED, "fused")]
K = len(CANDIDATES)
FUSED = 5
N_FEATURES = 16
DEFAULT_CHOICE = 1  # slabs at the natural width: the reference's own format
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_model.npz")


@dataclass
class OpSpec:
    kind: str
    sel: float = 1.0
    rhs_bits: int = 0
    groups: int = 0


@dataclass
class ChainSpec:
    n: int
    bits: int
    ops: list = field(default_factory=list)
    seed: int = 0


def random_chain(rng: np.random.Generator, seed: int, n_range=(16, 26)) -> ChainSpec:
    """Length uniform in 2..5, operators uniform, n log-uniform in [2^16, 2^26], width uniform in
    1..32, selectivities uniform in [0.01, 0.99], group cardinalities log-uniform in [2, 2^16]."""
    length = int(rng.integers(2, 6))
    n = int(math.exp(rng.uniform(n_range[0] * math.log(2), n_range[1] * math.log(2))))
    bits = int(rng.integers(1, 33))
    ops_ = []
    for _ in range(length):
        kind = OPS[int(rng.integers(0, len(OPS)))]
        ops_.append(OpSpec(kind, sel=float(rng.uniform(0.01, 0.99)), rhs_bits=int(rng.integers(1, 17)),
                           groups=int(math.exp(rng.uniform(math.log(2), 16 * math.log(2))))))
    return ChainSpec(n, bits, ops_, seed)


def natural_out_bits(kind: str, wx: int, wy: int) -> int:
    if kind == "add":
        return min(32, max(wx, wy) + 1)
    if kind == "mul":
        return min(32, wx + wy)
    return max(wx, wy)  # sub wraps modulo 2^width


def threshold(sel: float, w: int) -> int:
    """k of the predicate x < k for selectivity `sel` over a w-bit value range."""
    return max(1, int(round(sel * (1 << w))))


def key_bits(groups: int) -> int:
    return max(1, (groups - 1).bit_length())


def byte_bits(w: int) -> int:
    return 8 if w <= 8 else (16 if w <= 16 else 32)


@dataclass
class Point:
    """What the planner knows before operator i runs: the semantic width w and an upper bound
    on x's values, the estimated length, and the live mask (None without one): its share of
    passing elements and, while x is still the column it was computed on, the threshold that
    bounds the survivors' values."""
    w: int
    bound: int
    n_est: float
    mask_frac: float | None = None
    mask_k: int | None = None


def _pass_frac(bound: int, k: int) -> float:
    """Share of values uniform in [0, bound] below k."""
    return min(1.0, k / (bound + 1))


def _compress(pt: Point, sel: float) -> tuple:
    """(value bound, share of survivors) of a compressstore at pt."""
    if pt.mask_frac is None:
        k = threshold(sel, pt.w)
        return min(pt.bound, k - 1), _pass_frac(pt.bound, k)
    if pt.mask_k is not None:
        return min(pt.bound, pt.mask_k - 1), pt.mask_frac
    return pt.bound, pt.mask_frac


def candidate_valid(chain: ChainSpec, i: int, c: int) -> bool:
    """The fused variant exists only for a binary op whose result only a compressstore reads
    (directly, or through a filter right before it)."""
    if CANDIDATES[c][1] != "fused":
        return True
    ops_ = chain.ops
    if ops_[i].kind not in BINARY_OPS or i + 1 >= len(ops_):
        return False
    return ops_[i + 1].kind == "compressstore" or (
        ops_[i + 1].kind == "filter" and i + 2 < len(ops_) and ops_[i + 2].kind == "compressstore")


def candidate_storage(c: int, natural: int, bound: int) -> tuple:
    """(format, storage width) of candidate c for values of natural width `natural` bounded by
    `bound`; FORMAT_FUSED for the fused variant."""
    fmt, rule = CANDIDATES[c]
    if rule == "fused":
        return FORMAT_FUSED, natural
    if rule == "byte":
        return fmt, byte_bits(natural)
    if rule == "tight":
        return fmt, max(1, min(natural, int(bound).bit_length()))
    return fmt, natural


def hist_features(hist, w: int) -> tuple:
    """Two summaries of a column's bit-width histogram (hist[k] = values needing exactly k
    bits): the share of values that need at least w - 1 bits, and the share that need at most
    w / 2 bits."""
    h = np.asarray(hist, dtype=np.float64)
    tot = h.sum()
    if tot <= 0:
        return 0.0, 0.0
    top = h[max(0, w - 1):].sum() / tot
    low = h[: w // 2 + 1].sum() / tot
    return float(top), float(low)


def features(chain: ChainSpec, i: int, pt: Point, natural: int, bound: int, hist=None) -> np.ndarray:
    """16 features of decision point i: estimated length, widths (current, natural, tight,
    right operand), selectivity, position and remaining length, the consuming operator's kind,
    this operator's kind, the input column's bit-width histogram, and the cardinality of a later
    group-by."""
    op = chain.ops[i]
    nxt = chain.ops[i + 1].kind if i + 1 < len(chain.ops) else None
    later_groups = max([o.groups for o in chain.ops[i + 1:] if o.kind == "groupby"], default=0)
    f = np.zeros(N_FEATURES, np.float32)
    f[0] = math.log2(max(pt.n_est, 1.0)) / 26.0
    f[1] = pt.w / 32.0
    f[2] = natural / 32.0
    f[3] = max(1, int(bound).bit_length()) / 32.0
    f[4] = (op.rhs_bits / 32.0) if op.kind in BINARY_OPS else 0.0
    f[5] = _compress(pt, op.sel)[1] if op.kind == "compressstore" else 1.0
    f[6] = i / 5.0
    f[7] = (len(chain.ops) - 1 - i) / 5.0
    f[8] = 1.0 if nxt in ("filter", "compressstore") else 0.0
    f[9] = 1.0 if nxt in BINARY_OPS else 0.0
    f[10] = 1.0 if nxt in ("sum", "min", "max", "groupby") else 0.0
    f[12] = 1.0 if op.kind == "compressstore" else 0.0
    f[13] = 1.0 if op.kind == "mul" else 0.0
    if hist is not None:
        f[11], f[14] = hist_features(hist, chain.bits)
    f[15] = math.log2(later_groups) / 16.0 if later_groups else 0.0
    return f


def decision_points(chain: ChainSpec) -> list:
    return [i for i, o in enumerate(chain.ops) if o.kind in DECISION_OPS]


def valid_combos(chain: ChainSpec):
    """Every assignment of candidates to the decision points (the exhaustive sweep)."""
    import itertools

    dps = decision_points(chain)
    choices = [[c for c in range(K) if candidate_valid(chain, i, c)] for i in dps]
    return [tuple(x) for x in itertools.product(*choices)]


def plan(chain: ChainSpec, choose, hist=None):
    """Walks the chain, asking choose(i, feats, valid) -> candidate for every decision point
    (valid = the candidates that exist there), and returns the list of per-operator
    (kind, params) the executors turn into launches:
      ("filter", k) / ("compressstore", k, fmt, bits) / ("binary", op, value_bits, fmt, bits) /
      ("reduce", agg) / ("groupby",)
    plus the choices made."""
    pt = Point(chain.bits, (1 << chain.bits) - 1, float(chain.n))
    steps, choices = [], []
    for i, op in enumerate(chain.ops):
        if op.kind == "filter":
            k = threshold(op.sel, pt.w)
            steps.append(("filter", k))
            pt = Point(pt.w, pt.bound, pt.n_est, _pass_frac(pt.bound, k), k)
        elif op.kind == "compressstore":
            k = threshold(op.sel, pt.w)  # used only without a live mask
            nb, frac = _compress(pt, op.sel)
            valid = [c for c in range(K) if candidate_valid(chain, i, c)]
            c = choose(i, features(chain, i, pt, pt.w, nb, hist), valid)
            choices.append(c)
            fmt, sb = candidate_storage(c, pt.w, nb)
            steps.append(("compressstore", k, fmt, sb))
            pt = Point(pt.w, nb, pt.n_est * frac)
        elif op.kind in BINARY_OPS:
            ry = (1 << op.rhs_bits) - 1
            nat = natural_out_bits(op.kind, pt.w, op.rhs_bits)
            cap = (1 << nat) - 1
            if op.kind == "add":
                nb = min(pt.bound + ry, cap)
            elif op.kind == "mul":
                nb = min(pt.bound * ry, cap)
            else:
                nb = cap
            valid = [c for c in range(K) if candidate_valid(chain, i, c)]
            c = choose(i, features(chain, i, pt, nat, nb, hist), valid)
            choices.append(c)
            fmt, sb = candidate_storage(c, nat, nb)
            steps.append(("binary", BINARY_OPS[op.kind], nat, fmt, sb))
            # the mask stays live, but it no longer bounds the values of the new x
            pt = Point(nat, nb, pt.n_est, pt.mask_frac, None)
        elif op.kind in AGG_OPS:
            steps.append(("reduce", AGG_OPS[op.kind]))
        else:
            steps.append(("groupby",))
    return steps, choices


def fixed(c: int):
    """choose() that takes candidate c wherever it exists, else the default."""
    return lambda i, f, valid: c if c in valid else DEFAULT_CHOICE


def from_combo(combo):
    it = iter(combo)
    return lambda i, f, valid: next(it)


STEP_KINDS = {"filter": STEP_FILTER, "compressstore": STEP_COMPRESSSTORE, "binary": STEP_BINARY,
              "reduce": STEP_REDUCE, "groupby": STEP_GROUPBY}
