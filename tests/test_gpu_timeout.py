"""The failure path of the bounded device-side waits, made to run out without any fault or hang:
amx_test_lookback_timeout stops the kernel from publishing one tile's look-back count and
shortens every look-back poll loop, so the waits on that tile give up.  The kernel must record
AMX_ERR_TIMEOUT, finish, and leave the context usable: the same call without the hook is
bit-exact again.  (The reference prints and exits on any error, src/cuda_try.cuh:8-21.)"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import SLAB, gpu_bytes, make_column, to_gpu

pytestmark = pytest.mark.gpu

UNSET = (1 << 64) - 1


def test_lookback_wait_runs_out_and_is_reported(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import ops
    from oracle import oracle as O

    L = A.lib()
    n = 1 << 21  # hundreds of tiles, so other CTAs wait on tile 0
    v, raw = make_column(77, SLAB, 11, n)
    col = to_gpu(raw, n, SLAB, 11)
    p = ops.predicate(A.PRED_LT, 205, 0, 11)
    want, wcnt = O.filter_compressstore(raw, n, SLAB, 11, O.pred(A.PRED_LT, 205), SLAB, 11)
    ws = ops.workspace(n)
    try:
        A.check(L.amx_test_lookback_timeout(0, 2000))
        out, cnt = ops.filter_compressstore(col, p, SLAB, 11, ws=ws)
        st = L.amx_workspace_status(C.c_void_p(ws.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 6, A.lib().amx_last_error()
        assert int(cnt[0].item()) == wcnt  # the count comes from the CTA totals, not the look-back
    finally:
        L.amx_test_lookback_timeout(UNSET, 0)
    out, cnt = ops.filter_compressstore(col, p, SLAB, 11, ws=ws)
    ops.workspace_status(ws)
    assert int(cnt[0].item()) == wcnt
    assert np.array_equal(gpu_bytes(out, wcnt), want)


def test_program_reports_a_step_timeout(cuda):
    """A chain program whose compressstore's look-back runs out reports it through
    amx_program_status; the rerun without the hook is clean."""
    from amethyst_b200 import _capi as A
    from amethyst_b200 import chains as X
    from amethyst_b200 import selector as S

    L = A.lib()
    ch = X.ChainSpec(1 << 20, 13, [X.OpSpec("add", rhs_bits=9), X.OpSpec("compressstore", sel=0.4), X.OpSpec("sum")], 3)
    r = S.ChainRunner(ch)
    prog, _ = r.program(X.fixed(X.DEFAULT_CHOICE))
    try:
        A.check(L.amx_test_lookback_timeout(0, 2000))
        prog.run()
        with pytest.raises(A.AmxError) as e:
            prog.status()
        assert e.value.status == 6
    finally:
        L.amx_test_lookback_timeout(UNSET, 0)
    prog.run()
    prog.status()
