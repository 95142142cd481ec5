"""Grouped point search at batch sizes that take the staged-window kernel
(2^21 queries and more): bit-exact against the CPU oracle for every key and
value width, search configuration and key distribution that moves the window
to another separator level, and for input that is not grouped at all."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NQ = (1 << 21) + 77  # above the window kernel's batch threshold, ragged tail


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def batch(keys, kt, g, nq=NQ):
    hi = int(np.iinfo(kt).max)
    q = np.concatenate([keys[g.integers(0, len(keys), size=nq // 2)],
                        g.integers(0, hi, size=nq - nq // 2 - 4, dtype=np.uint64,
                                   endpoint=True).astype(kt),
                        np.array([0, 1, hi, hi - 1], dtype=kt)])
    g.shuffle(q)
    return q


def keys_of(kind, n, kt, g):
    hi = int(np.iinfo(kt).max)
    if kind == "uniform":
        k = g.integers(0, hi, size=n + n // 8 + 16, dtype=np.uint64, endpoint=True)
    elif kind == "narrow":  # every key in one group: the window moves up the tree
        k = g.integers(0, 1 << 22, size=n + n // 8 + 16, dtype=np.uint64)
    else:  # half the keys in one group, the rest spread
        k = np.concatenate([g.integers(0, hi, size=n // 2, dtype=np.uint64, endpoint=True),
                            (hi >> 1) + g.integers(0, 1 << 20, size=n, dtype=np.uint64)])
    return np.unique(k)[:n].astype(kt)


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint32, np.uint64),
                                   (np.uint64, np.uint32), (np.uint64, np.uint64)])
@pytest.mark.parametrize("kind", ["uniform", "narrow", "skewed"])
def test_grouped_window_exact(bt, orc, cuda, kt, vt, kind):
    g = np.random.default_rng(hash((np.dtype(kt).itemsize, np.dtype(vt).itemsize, kind)) & 0xFFFF)
    keys = keys_of(kind, 1 << 22, kt, g)
    vals = g.integers(0, int(np.iinfo(vt).max), size=len(keys), dtype=np.uint64).astype(vt)
    q = batch(keys, kt, g)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        dq = dev(q, cuda)
        assert np.array_equal(t.point_search(dq, mode="grouped").cpu().numpy(), exp)
        grouped, perm = t.group(dq)
        assert np.array_equal(t.search_grouped_batch(grouped, perm).cpu().numpy(), exp)


@pytest.mark.parametrize("cfg", [(8, 1), (8, 2), (4, 1), (4, 2), (2, 1)])
def test_grouped_window_every_config(bt, orc, cuda, cfg):
    g = np.random.default_rng(cfg[0] * 10 + cfg[1])
    keys = keys_of("uniform", 3 << 20, np.uint32, g)
    vals = np.arange(len(keys), dtype=np.uint32)
    q = batch(keys, np.uint32, g)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        t.set_search_config(*cfg)
        assert np.array_equal(t.point_search(dev(q, cuda), mode="grouped").cpu().numpy(), exp)


@pytest.mark.parametrize("n", [1, 37, 5000, 300001])
def test_grouped_window_small_trees(bt, orc, cuda, n):
    g = np.random.default_rng(n)
    keys = keys_of("uniform", n, np.uint32, g)
    vals = np.arange(len(keys), dtype=np.uint32)
    q = batch(keys, np.uint32, g)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        assert np.array_equal(t.point_search(dev(q, cuda), mode="grouped").cpu().numpy(), exp)


def test_grouped_batch_accepts_ungrouped_input(bt, orc, cuda):
    """Input in random order with an identity permutation: every tile mixes
    groups, so the kernel must take the full descent and stay exact."""
    import torch
    g = np.random.default_rng(7)
    keys = keys_of("uniform", 1 << 22, np.uint32, g)
    vals = np.arange(len(keys), dtype=np.uint32)
    q = batch(keys, np.uint32, g)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        perm = torch.arange(len(q), dtype=torch.int64, device=cuda).to(torch.uint32)
        got = t.search_grouped_batch(dev(q, cuda), perm).cpu().numpy()
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("kt", [np.uint32, np.uint64])
def test_grouped_window_tiny_key_range(bt, orc, cuda, kt):
    """Keys 0..199: groups are single key values (the group shift is 0), the
    last group holds every larger query."""
    g = np.random.default_rng(200)
    keys = np.arange(0, 200, dtype=kt)
    vals = g.permutation(200).astype(kt)
    q = g.integers(0, 300, size=NQ, dtype=np.uint64).astype(kt)
    q[:4] = [0, 199, 200, np.iinfo(kt).max]
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        assert np.array_equal(t.point_search(dev(q, cuda), mode="grouped").cpu().numpy(), exp)
