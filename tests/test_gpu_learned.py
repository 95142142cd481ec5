"""Learned index: the root's gradient kernel, the segmentation against the
oracle's restatement, exact search, and what training buys."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHUNK = 1 << 14  # keys per segmentation thread (a segment never crosses a multiple)
HULL_CAP = 32


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


def queries_for(keys, g, kt, nhit=40000, nrand=20000):
    return np.concatenate([keys[g.integers(0, len(keys), size=nhit)],
                           g.integers(0, int(keys[-1]) + 2, size=nrand, dtype=np.uint64).astype(kt),
                           (keys[:2000].astype(np.uint64) + 1).astype(kt),
                           (keys[-2000:].astype(np.uint64) - 1).astype(kt),
                           np.array([0, np.iinfo(kt).max, keys[0], keys[-1]], dtype=kt)])


@pytest.mark.parametrize("kind,n,kt,vt,target", [
    ("lognormal", 1 << 20, np.uint64, np.uint64, {"num_segments": 1024}),
    ("lognormal", 1 << 20, np.uint64, np.uint64, {"max_error": 16}),
    ("lognormal", 300001, np.uint64, np.uint32, {"max_error": 64}),
    ("uniform", 1 << 20, np.uint32, np.uint32, {"num_segments": 4096}),
    ("uniform", 70001, np.uint32, np.uint64, {"max_error": 4}),
    ("uniform", 2, np.uint64, np.uint64, {"max_error": 1}),
    ("uniform", 37, np.uint32, np.uint32, {"max_error": 1}),
    ("uniform", 5000, np.uint64, np.uint64, {"num_segments": 3}),
    ("uniform", 65536 * 8 + 3, np.uint64, np.uint64, {"max_error": 2}),
])
def test_learned_search_is_exact(bt, orc, cuda, kind, n, kt, vt, target):
    g = np.random.default_rng(n)
    if kind == "lognormal":
        keys = lognormal_keys(n).astype(kt)
    else:
        keys = np.unique(g.integers(0, np.iinfo(kt).max, size=n + n // 8 + 8,
                                    dtype=np.uint64))[:n].astype(kt)
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    q = queries_for(keys, g, kt)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        rep = t.learned_train(iterations=200, **target)
        assert rep["root_loss_final"] <= rep["root_loss_initial"] + 1e-6
        if "max_error" in target:
            assert rep["max_error"] == target["max_error"]
        else:
            assert rep["num_segments"] <= target["num_segments"]
        for shape in (1, 2, 3, 4):  # kernel shapes
            t.learned_set_shape(shape)
            got = t.point_search_learned(dev(q, cuda)).cpu().numpy()
            assert np.array_equal(got, exp), shape
            extra, fallback = t.learned_last_stats()
            assert 0 <= t.learned_last_lines() <= 4 * len(q)
            assert fallback == 0  # the measured bounds always hold
            assert extra <= len(q) // 20
        for bad in (0, 5):
            with pytest.raises(bt.BTreeError):
                t.learned_set_shape(bad)


def test_learned_with_duplicate_keys(bt, orc, cuda):
    """Runs of equal keys (the tree keeps them): the first occurrence's value."""
    g = np.random.default_rng(9)
    keys = np.sort(np.repeat(g.integers(0, 1 << 40, size=20000, dtype=np.uint64),
                             g.integers(1, 40, size=20000)))
    vals = np.arange(len(keys), dtype=np.uint64)
    q = np.concatenate([keys[g.integers(0, len(keys), size=30000)],
                        g.integers(0, 1 << 40, size=10000, dtype=np.uint64)])
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        for eps in (1, 8, 100):
            t.learned_train(max_error=eps, iterations=100)
            assert np.array_equal(t.point_search_learned(dev(q, cuda)).cpu().numpy(), exp), eps
            assert t.learned_last_stats()[1] == 0


@pytest.mark.parametrize("n,eps", [(1 << 20, 16), (1 << 20, 64), (3 * CHUNK + 77, 8)])
def test_segmentation_matches_the_oracle(bt, orc, cuda, n, eps):
    """The GPU segmentation has exactly the segments of the oracle's
    restatement (same chunking and hull cap)."""
    keys = lognormal_keys(n, seed=n)
    exp = orc.pla_segments(keys, eps, chunk=CHUNK, hull_cap=HULL_CAP, lines=False)
    with bt.Tree.build(dev(keys, cuda), dev(np.arange(n, dtype=np.uint64), cuda)) as t:
        rep = t.learned_train(max_error=eps, iterations=10)
    assert rep["num_segments"] == exp
    # FP32 rounding of the lines can only add a rank or two to the bound
    assert rep["eps_max"] <= eps + 2


def test_segment_target_picks_the_least_bound(bt, orc, cuda):
    keys = lognormal_keys(1 << 20, seed=4)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        rep = t.learned_train(num_segments=512, iterations=10)
    eps = rep["max_error"]
    assert rep["num_segments"] <= 512
    assert orc.pla_segments(keys, eps, chunk=CHUNK, hull_cap=HULL_CAP, lines=False) <= 512
    assert orc.pla_segments(keys, eps - 1, chunk=CHUNK, hull_cap=HULL_CAP, lines=False) > 512


def test_too_many_segments_is_refused(bt, cuda):
    keys = lognormal_keys(1 << 20, seed=6)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        with pytest.raises(bt.BTreeError) as e:
            t.learned_train(max_error=1, iterations=1)  # ~2^19 segments
        assert e.value.name == "BT_ERR_NOT_SUPPORTED"


def test_learned_requires_a_trained_model(bt, cuda):
    keys = np.arange(100, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        with pytest.raises(bt.BTreeError):
            t.point_search_learned(dev(keys, cuda))


def test_training_gains_over_the_untrained_network(bt, orc, cuda):
    """What the root network buys.  Without it, each query would binary-search
    all the segment lines' first keys (log2(lines) probes); the untrained
    network (ramps forming the identity) narrows that to 2 e + 3 of them for
    its worst error e over those keys; training narrows it further."""
    keys = lognormal_keys(1 << 22, seed=5)
    vals = np.arange(len(keys), dtype=np.uint64)
    g = np.random.default_rng(3)
    q = keys[g.integers(0, len(keys), size=1 << 18)]
    exp = orc.point_search(keys, vals, q)
    res = {}
    for iters in (0, 600):
        with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
            rep = t.learned_train(num_segments=1 << 14, iterations=iters)
            assert np.array_equal(t.point_search_learned(dev(q, cuda)).cpu().numpy(), exp)
            assert t.learned_last_stats()[1] == 0
            res[iters] = rep
    untrained, trained = res[0], res[600]
    assert untrained["root_error"] == untrained["root_error_initial"]
    assert trained["root_loss_final"] < untrained["root_loss_final"]
    assert trained["root_error"] <= untrained["root_error"]
    lines = (trained["num_segments"] + 3) // 4
    steps = lambda e: np.ceil(np.log2(min(2 * e + 3, lines)))
    assert steps(trained["root_error"]) < np.ceil(np.log2(lines))
