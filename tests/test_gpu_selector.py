"""The selector network's CUDA kernels against a plain PyTorch FP32 reference (forward and one
Adam training step, tolerance 1e-5 / 1e-4), training to a separable toy target, and the label
sweep and exhaustive judge over replayed chain graphs (chain results: test_gpu_program.py)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def torch_forward(p, x, K):
    import torch

    W1 = p[:1024].view(64, 16)
    b1 = p[1024:1088]
    W2 = p[1088:5184].view(64, 64)
    b2 = p[5184:5248]
    W3 = p[5248:5248 + 64 * K].view(K, 64)
    b3 = p[5248 + 64 * K:5248 + 65 * K]
    h1 = torch.relu(x @ W1.T + b1)
    h2 = torch.relu(h1 @ W2.T + b2)
    return h2 @ W3.T + b3


def test_forward_matches_torch(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import selector as S

    for K in (2, 4, 8):
        g = torch.Generator().manual_seed(K)
        p = (torch.rand(int(A.lib().amx_mlp_param_count(K)), generator=g) - 0.5).cuda()
        x = torch.rand(1000, 16, generator=g).cuda()
        probs = torch.empty(1000, K, device="cuda")
        A.check(A.lib().amx_mlp_forward(C.c_void_p(p.data_ptr()), K, C.c_void_p(x.data_ptr()), 1000,
                                        C.c_void_p(probs.data_ptr()), None))
        torch.cuda.synchronize()
        want = torch.softmax(torch_forward(p, x, K), dim=1)
        assert torch.allclose(probs, want, atol=1e-5, rtol=1e-5)
    assert S.K == 6


def test_train_step_matches_torch_adam(cuda):
    import torch

    from amethyst_b200 import _capi as A
    from amethyst_b200 import selector as S

    K, B = S.K, 64
    p0 = torch.from_numpy(S.init_params(3)).cuda()
    g = torch.Generator().manual_seed(5)
    x = torch.rand(B, 16, generator=g).cuda()
    y = torch.randint(0, K, (B,), generator=g).to(torch.int32).cuda()
    p = p0.clone()
    adam = torch.zeros(2 * p.numel(), device="cuda")
    loss = torch.zeros(1, device="cuda")
    for step in (1, 2):
        A.check(A.lib().amx_mlp_train_step(C.c_void_p(p.data_ptr()), C.c_void_p(adam.data_ptr()), step, K,
                                           C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), B, C.c_float(1e-2),
                                           C.c_void_p(loss.data_ptr()), None))
    torch.cuda.synchronize()
    q = p0.clone().requires_grad_(True)
    opt = torch.optim.Adam([q], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    for _ in range(2):
        opt.zero_grad()
        l = torch.nn.functional.cross_entropy(torch_forward(q, x, K), y.long())
        l.backward()
        opt.step()
    assert torch.allclose(p, q.detach(), atol=1e-5, rtol=1e-4)
    assert abs(float(loss.item()) - float(l.item())) < 1e-4 * max(1.0, abs(float(l.item())))


def test_training_learns_a_separable_target(cuda):
    from amethyst_b200 import selector as S

    rng = np.random.default_rng(1)
    x = rng.random((4000, 16), dtype=np.float32)
    w = rng.standard_normal((16, S.K)).astype(np.float32)
    y = (x @ w).argmax(1).astype(np.uint32)
    params, hist = S.train(x[:3500], y[:3500], epochs=40)
    acc = (S.Selector(params).probs(x[3500:]).argmax(1) == y[3500:]).mean()
    assert hist[-1] < hist[0] and acc > 0.9, (hist[0], hist[-1], acc)


def test_sweep_and_exhaustive_shapes(cuda):
    from amethyst_b200 import selector as S

    rng = np.random.default_rng(3)
    ch = S.random_chain(rng, seed=77, n_range=(14, 15))
    ch.ops = [S.OpSpec("compressstore", sel=0.3), S.OpSpec("add", rhs_bits=5), S.OpSpec("sum")]
    f, l, t = S.sweep_labels(ch, reps=1)
    assert f.shape == (2, 16) and l.shape == (2,) and t.shape == (2, S.K)
    assert all(int(l[i]) == int(np.argmin(t[i])) for i in range(2))
    assert np.isinf(t[:, S.FUSED]).all()  # no binary op feeds a compressstore here
    best, combo, table = S.exhaustive(ch, reps=1)
    assert len(table) == (S.K - 1) ** 2 and best == min(table.values())
    ch.ops = [S.OpSpec("mul", rhs_bits=3), S.OpSpec("compressstore", sel=0.4), S.OpSpec("max")]
    f, l, t = S.sweep_labels(ch, reps=1)
    assert np.isfinite(t[0, S.FUSED]) and np.isinf(t[1, S.FUSED])


def test_selector_picks_valid_candidates(cuda):
    from amethyst_b200 import chains as X
    from amethyst_b200 import selector as S

    sel = S.Selector(S.init_params(5))
    rng = np.random.default_rng(8)
    runners = [S.ChainRunner(X.random_chain(rng, seed=900 + k, n_range=(10, 12))) for k in range(12)]
    picks = sel.choices(runners)
    for r, p in zip(runners, picks):
        dps = X.decision_points(r.chain)
        assert len(p) == len(dps)
        assert all(X.candidate_valid(r.chain, i, c) for i, c in zip(dps, p))
