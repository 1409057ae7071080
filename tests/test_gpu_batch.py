"""One-launch batches of slab columns (filter + compressstore + sum) against the C oracle per
column, bit-exact, through the C ABI: uneven lengths (including empty columns and tile edges),
every width 1..32, edge predicates, both block shapes, and replay from a captured CUDA graph."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import SLAB, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu


def build(seed, ncols, max_n=300000):
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    rng = np.random.default_rng(seed)
    cols, preds, raws, want = [], [], [], []
    kinds = [A.PRED_LT, A.PRED_GE, A.PRED_BETWEEN, A.PRED_NOT_BETWEEN, A.PRED_NE, A.PRED_ALL, A.PRED_GT]
    for i in range(ncols):
        bits = int(rng.integers(1, 33)) if i >= 32 else i + 1
        n = int([0, 1, 2, 63, 64, 65, 4095, 16384, 16385][i % 9] if i % 3 == 0 else rng.integers(1, max_n))
        v, raw = make_column(seed * 1000 + i, SLAB, bits, n)
        top = (1 << bits) - 1
        kind = kinds[i % len(kinds)]
        k0 = int(rng.integers(0, top + 1))
        k1 = int(rng.integers(k0, top + 1))
        p = ops.predicate(kind, k0, k1, bits)
        cols.append(to_gpu(raw, n, SLAB, bits))
        preds.append(p)
        raws.append(raw)
        want.append(O.chain(A.OP_LHS, (raw, SLAB, bits), None, bits, O.pred(kind, k0, k1, bits), A.AGG_SUM, SLAB,
                            bits, n))
    return cols, preds, want


def check(batch, want):
    counts = batch.counts.cpu().numpy().view(np.uint64)
    sums = batch.sums.cpu().numpy().view(np.uint64)
    for i, (wout, wcnt, wsum) in enumerate(want):
        assert int(counts[i]) == wcnt, (i, batch.cols[i].n, batch.cols[i].bits)
        assert int(sums[i]) == wsum, i
        assert np.array_equal(gpu_bytes(batch.outs[i], wcnt), wout), (i, batch.cols[i].n, batch.cols[i].bits)


@pytest.mark.parametrize("threads,wpt", [(256, 8), (512, 8), (256, 3), (512, 1), (256, 2), (512, 5)])
def test_batch_matches_oracle(cuda, threads, wpt):
    """Every block shape and tile size (slab words per thread) the autotuner may pick."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    cols, preds, want = build(threads + wpt, 70)
    b = ops.Batch(cols, preds, A.BatchTuning(threads, 0, wpt))
    b.run()
    check(b, want)
    b.run()  # a second run on the same plan and workspace
    check(b, want)
    b.status()


def test_batch_graph_replay(cuda):
    import torch

    from amethyst_b200 import ops

    cols, preds, want = build(7, 40)
    b = ops.Batch(cols, preds)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.run(s)  # warm-up outside capture
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(s)
    for o in b.outs:
        o.data.zero_()
    b.counts.zero_()
    g.replay()
    torch.cuda.synchronize()
    check(b, want)


def test_batch_empty(cuda):
    from amethyst_b200 import ops

    b = ops.Batch([], [])
    b.run()
    b.status()
