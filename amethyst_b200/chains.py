"""Operator chains for the format selector: the synthetic chain distribution, the storage
candidates of a decision point, and the 16 features the selector network reads.  Host logic only
(no torch, no GPU), shared by the selector and its CPU tests."""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from ._capi import NOGAPS, PLAIN32, SLAB

OPS = ["filter", "compressstore", "add", "sub", "mul", "sum", "min", "max", "groupby"]
DECISION_OPS = {"compressstore", "add", "sub", "mul"}
CANDIDATES = [(PLAIN32, "natural"), (SLAB, "natural"), (SLAB, "byte"), (NOGAPS, "natural")]
K = len(CANDIDATES)
N_FEATURES = 16
DEFAULT_CHOICE = 1  # slabs at the natural width
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


def candidate_bits(c: int, w: int, kind: str = "") -> int:
    """Storage width of candidate c for values of natural width w.  A subtraction wraps modulo
    2^width, so it is always stored at its natural width (its byte candidate equals candidate 1)."""
    if CANDIDATES[c][1] == "byte" and kind != "sub":
        return 8 if w <= 8 else (16 if w <= 16 else 32)
    return w


def features(chain: ChainSpec, i: int, n_cur: int, w_cur: int, out_w: int) -> np.ndarray:
    """16 features of decision point i: current length, widths, selectivity, position and
    remaining length, the kind of operator that reads the output, this operator's kind, and the
    group cardinality of a later group-by."""
    op = chain.ops[i]
    nxt = chain.ops[i + 1].kind if i + 1 < len(chain.ops) else None
    later_groups = max([o.groups for o in chain.ops[i + 1:] if o.kind == "groupby"], default=0)
    f = np.zeros(N_FEATURES, np.float32)
    f[0] = math.log2(max(n_cur, 1)) / 26.0
    f[1] = w_cur / 32.0
    f[2] = out_w / 32.0
    f[3] = (op.rhs_bits / 32.0) if op.kind in ("add", "sub", "mul") else 0.0
    f[4] = op.sel if op.kind == "compressstore" else 1.0
    f[5] = i / 5.0
    f[6] = (len(chain.ops) - 1 - i) / 5.0
    f[7] = 1.0 if nxt in ("filter", "compressstore") else 0.0
    f[8] = 1.0 if nxt in ("add", "sub", "mul") else 0.0
    f[9] = 1.0 if nxt in ("sum", "min", "max") else 0.0
    f[10] = 1.0 if nxt == "groupby" else 0.0
    f[11] = 1.0 if nxt is None else 0.0
    f[12] = 1.0 if op.kind == "compressstore" else 0.0
    f[13] = 1.0 if op.kind in ("add", "sub") else 0.0
    f[14] = 1.0 if op.kind == "mul" else 0.0
    f[15] = math.log2(later_groups) / 16.0 if later_groups else 0.0
    return f


