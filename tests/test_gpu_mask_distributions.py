"""Compressstore and masked aggregation under the reference's own mask distributions: uniform,
one cluster and eight clusters of set bits at selectivities 0.01 .. 0.9 (the generators of
src/main.cu:33-108 as run by src/run.sh:6-22, restated in the oracle and pinned against the
reference's host code by tests/test_golden.py).  Bit-exact against the oracle and, when the
reference's kernels are built, against its popcount -> CUB scan -> write pipeline."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import SLAB, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu

N = 1 << 20
SELECTIVITIES = [0.01, 0.1, 0.25, 0.5, 0.9]


def masks(sel):
    return {
        "uniform": O.mask_uniform(((N + 63) // 64) * 8, sel)[: N // 8],
        "one_cluster": O.mask_clusters(sel, 1, N),
        "eight_clusters": O.mask_clusters(sel, 8, N),
    }


@pytest.mark.parametrize("sel", SELECTIVITIES)
@pytest.mark.parametrize("bits", [3, 11, 32])
def test_compressstore_under_reference_masks(cuda, sel, bits):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops

    _, raw = make_column(int(sel * 1000) + bits, SLAB, bits, N)
    col = to_gpu(raw, N, SLAB, bits)
    ref = O.ref_gpu()
    for name, m8 in masks(sel).items():
        m = np.zeros(N // 32 + 4, np.uint32)
        m[: N // 32] = m8.view(np.uint32)
        dm = torch.from_numpy(m.view(np.int32)).cuda()
        out, cnt = ops.compressstore(col, dm, SLAB, bits)
        want, wcnt = O.compressstore(raw, N, SLAB, bits, m[: N // 32], SLAB, bits)
        assert int(cnt[0].item()) == wcnt, (name, sel, bits)
        assert np.array_equal(gpu_bytes(out, wcnt), want), (name, sel, bits)
        s = int(ops.hop(A.AGG_SUM, col, dm).cpu().numpy().view(np.uint64)[0])
        assert s == O.reduce(A.AGG_SUM, raw, N, SLAB, bits, m[: N // 32]), (name, sel, bits)
        if ref is not None:
            pad = 1 << 20
            d = torch.zeros(len(raw) + pad, dtype=torch.uint8, device="cuda")
            d[: len(raw)].copy_(torch.from_numpy(raw.copy()))
            rm = torch.zeros(N // 8 + pad, dtype=torch.uint8, device="cuda")
            rm[: N // 8].copy_(torch.from_numpy(m8.copy()))
            rout = torch.zeros(len(raw) + pad, dtype=torch.uint8, device="cuda")
            rc = C.c_uint64(0)
            assert ref.amxref_gpu_compressstore_slabs(bits, C.c_void_p(rm.data_ptr()), C.c_void_p(d.data_ptr()),
                                                      C.c_void_p(rout.data_ptr()), N, C.byref(rc), 1024) == 0
            assert rc.value == wcnt
            nb = O.storage_bytes(SLAB, bits, wcnt)
            assert np.array_equal(O.decode(rout[:nb].cpu().numpy(), wcnt, SLAB, bits),
                                  O.decode(gpu_bytes(out, wcnt), wcnt, SLAB, bits)), (name, sel, bits)
