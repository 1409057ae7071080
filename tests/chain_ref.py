"""The chain semantics of amethyst_b200.chains run on the C oracle, operator by operator, over
host copies of a ChainRunner's columns: the checker for programs, graphs and the plain
per-operator form.  Every intermediate is kept in slabs at its natural width, as the plain form
does; the oracle's operators are the ones the per-operator parity tests pin to the reference."""
from __future__ import annotations

import numpy as np

from amethyst_b200 import chains as X
from oracle import oracle as O

SLAB = 2


def host_column(col):
    """(raw bytes, format, bits, n) of a device PackedColumn."""
    nb = O.storage_bytes(col.fmt, col.bits, col.n)
    raw = np.zeros(nb + 16, np.uint8)
    raw[:nb] = col.data[:nb].cpu().numpy()
    return raw, col.fmt, col.bits, col.n


def run(runner) -> list:
    """The digest ChainRunner.digest would give for a correct run of the chain."""
    ch = runner.chain
    steps, _ = X.plan(ch, X.fixed(X.DEFAULT_CHOICE))
    raw, fmt, bits, n = host_column(runner.x0)
    mask = None
    res = [0] * len(ch.ops)
    groups = []
    for i, st in enumerate(steps):
        kind = st[0]
        if kind == "filter":
            mask = O.filter(raw, n, fmt, bits, O.pred(1, st[1]))
        elif kind == "compressstore":
            if mask is not None:
                out, cnt = O.compressstore(raw, n, fmt, bits, mask, st[2], st[3])
            else:
                out, cnt = O.filter_compressstore(raw, n, fmt, bits, O.pred(1, st[1]), st[2], st[3])
            raw = np.concatenate([out, np.zeros(16, np.uint8)])
            fmt, bits, n = st[2], st[3], cnt
            res[i] = cnt
            mask = None
        elif kind == "binary":
            araw, afmt, abits, _ = host_column(runner.aux[i])
            out = O.binary(st[1], raw, fmt, bits, araw, afmt, abits, n, st[3], st[4])
            raw = np.concatenate([out, np.zeros(16, np.uint8)])
            fmt, bits = st[3], st[4]
        elif kind == "reduce":
            res[i] = O.reduce(st[1], raw, n, fmt, bits, mask)
        else:
            kraw, kfmt, kbits, _ = host_column(runner.aux[i])
            kn = n
            vraw, vfmt, vbits = raw, fmt, bits
            if mask is not None:
                kout, kn = O.compressstore(kraw, n, kfmt, kbits, mask, SLAB, kbits)
                vout, _ = O.compressstore(raw, n, fmt, bits, mask, SLAB, bits)
                kraw, kfmt = np.concatenate([kout, np.zeros(16, np.uint8)]), SLAB
                vraw, vfmt = np.concatenate([vout, np.zeros(16, np.uint8)]), SLAB
            g, sums, counts = O.groupby_dense(kraw, kfmt, kbits, vraw, vfmt, vbits, kn)
            present = np.nonzero(counts)[0]
            res[i] = int(g)
            groups.append(("g", i, int(g), present.astype(np.uint32).tobytes(), sums[present].astype(np.uint64).tobytes(),
                           counts[present].astype(np.uint64).tobytes()))
    out = [("r", [int(v) & 0xFFFFFFFFFFFFFFFF for v in res])] + groups
    if n:
        vals = O.decode(raw, n, fmt, bits).astype(np.uint64)
        out.append(("c", n, vals.tobytes()))
    else:
        out.append(("c", 0))
    return out
