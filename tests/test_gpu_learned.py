"""Learned position model: gradient check, exact search, and what training buys."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


@pytest.mark.parametrize("H", [1, 4, 16, 32])
def test_mlp_gradient_kernel_matches_cpu(bt, cuda, H):
    """The GPU forward/backward kernel against the CPU reference (float64)."""
    import torch
    from oracle import mlp_oracle as mo
    g = np.random.default_rng(H)
    n = 5000
    p = g.normal(0, 0.5, size=3 * H + 1).astype(np.float32)
    x = g.random(n).astype(np.float32)
    y = np.sort(g.random(n)).astype(np.float32)
    loss_d = torch.zeros(1, dtype=torch.float32, device=cuda)
    grad_d = torch.zeros(3 * H + 1, dtype=torch.float32, device=cuda)
    P = ctypes.c_void_p
    dp, dx, dy = dev(p, cuda), dev(x, cuda), dev(y, cuda)  # keep the buffers alive
    st = bt.lib().bt_mlp_loss_grad(P(dp.data_ptr()), H, P(dx.data_ptr()), P(dy.data_ptr()), n,
                                   P(loss_d.data_ptr()), P(grad_d.data_ptr()),
                                   P(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    l_cpu, g_cpu = mo.loss_grad(p, H, x, y)
    # the CPU analytic gradient itself agrees with finite differences
    assert np.allclose(g_cpu, mo.finite_diff_grad(p, H, x, y), rtol=1e-4, atol=1e-6)
    assert abs(loss_d.item() - l_cpu) <= 1e-4 * max(1.0, l_cpu)
    assert np.allclose(grad_d.cpu().numpy(), g_cpu, rtol=2e-3, atol=2e-5)


def lognormal_keys(n, seed=1):
    g = np.random.default_rng(seed)
    return np.cumsum(np.floor(g.lognormal(4.0, 2.0, size=n)).astype(np.uint64) + 1)


@pytest.mark.parametrize("kind,n,kt,vt", [
    ("lognormal", 1 << 20, np.uint64, np.uint64),
    ("lognormal", 300001, np.uint64, np.uint32),
    ("uniform", 1 << 20, np.uint32, np.uint32),
    ("uniform", 70001, np.uint32, np.uint64),
    ("uniform", 2, np.uint64, np.uint64),
    ("uniform", 37, np.uint32, np.uint32),
    ("uniform", 5000, np.uint64, np.uint64),
])
def test_learned_search_is_exact(bt, orc, cuda, kind, n, kt, vt):
    g = np.random.default_rng(n)
    if kind == "lognormal":
        keys = lognormal_keys(n).astype(kt)
    else:
        keys = np.unique(g.integers(0, np.iinfo(kt).max, size=n + n // 8 + 8,
                                    dtype=np.uint64))[:n].astype(kt)
    vals = np.arange(len(keys), dtype=vt)
    q = np.concatenate([keys[g.integers(0, len(keys), size=40000)],
                        g.integers(0, int(keys[-1]) + 2, size=20000, dtype=np.uint64).astype(kt),
                        (keys[:2000].astype(np.uint64) + 1).astype(kt),
                        np.array([0, np.iinfo(kt).max], dtype=kt)])
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        rep = t.learned_train(num_segments=min(65536, max(1, len(keys) // 16)), iterations=200)
        assert rep["root_loss_final"] <= rep["root_loss_initial"] + 1e-6
        for cfg in t.SEARCH_CONFIGS:
            t.set_search_config(*cfg)
            got = t.point_search_learned(dev(q, cuda)).cpu().numpy()
            assert np.array_equal(got, exp), cfg
        w, f = t.learned_last_stats()
        assert w + f == len(q)


def test_learned_requires_a_trained_model(bt, cuda):
    keys = np.arange(100, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        with pytest.raises(bt.BTreeError):
            t.point_search_learned(dev(keys, cuda))


def test_training_gains_over_the_untrained_network(bt, orc, cuda):
    """What the trained root buys over the same network untrained: a lower
    fit loss, tighter per-segment error bounds, narrower scan windows and far
    fewer queries that need the full descent."""
    keys = lognormal_keys(1 << 22, seed=5)
    vals = np.arange(len(keys), dtype=np.uint64)
    g = np.random.default_rng(3)
    q = keys[g.integers(0, len(keys), size=1 << 18)]
    exp = orc.point_search(keys, vals, q)
    res = {}
    for iters in (0, 400):
        with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
            rep = t.learned_train(num_segments=1 << 14, iterations=iters)
            got = t.point_search_learned(dev(q, cuda)).cpu().numpy()
            assert np.array_equal(got, exp)
            res[iters] = (rep, t.learned_last_stats())
    untrained, trained = res[0], res[400]
    assert trained[0]["root_loss_final"] < 0.1 * untrained[0]["root_loss_final"]
    assert trained[0]["eps_mean"] < untrained[0]["eps_mean"]
    assert trained[0]["window_lines_mean"] <= untrained[0]["window_lines_mean"]
    assert trained[1][1] <= untrained[1][1]
