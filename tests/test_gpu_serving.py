"""Continuous-batching request loop: results alone vs in the mix, overlap,
admission by device memory, request splitting."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t.numpy()


def requests(keys, g, count, max_size):
    out = []
    for _ in range(count):
        m = int(round(2 ** g.uniform(0, np.log2(max_size))))
        q = g.integers(0, int(keys[-1]) + 2, size=m, dtype=np.uint64).astype(keys.dtype)
        q[::2] = keys[g.integers(0, len(keys), size=len(q[::2]))]
        out.append(pinned(q))
    return out


@pytest.mark.parametrize("mode", ["basic", "grouped", "learned"])
def test_results_same_alone_and_mixed(bt, orc, cuda, mode):
    g = np.random.default_rng(11)
    keys = np.cumsum(np.floor(g.lognormal(4.0, 2.0, size=1 << 20)).astype(np.uint64) + 1)
    vals = np.arange(len(keys), dtype=np.uint64)
    reqs = requests(keys, g, 200, 1 << 14)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        if mode == "learned":
            t.learned_train(num_segments=1 << 14, iterations=200)
        with bt.Server(t, mode=mode, slots=8) as srv:
            alone = []
            for q in reqs:  # one at a time
                tk, out = srv.submit(q)
                srv.wait(tk)
                alone.append(out.copy())
            # all at once, with Poisson arrivals
            arr = np.cumsum(g.exponential(20.0, size=len(reqs)))
            lat, wall, mixed = srv.replay(reqs, arr)
            st = srv.stats()
        assert st["max_in_flight"] > 1, "requests never overlapped on the device"
        for q, a, m in zip(reqs, alone, mixed):
            exp = orc.point_search(keys, vals, q)
            assert np.array_equal(a, exp)
            assert np.array_equal(m, a)
        assert (lat > 0).all() and wall > 0


def test_memory_budget_limits_slots_and_large_requests_split(bt, orc, cuda):
    keys = np.arange(0, 3_000_000, 3, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        per_slot = 4096 * 8 + 512
        with bt.Server(t, slots=16, memory_budget_bytes=3 * per_slot, max_batch=4096) as srv:
            assert srv.stats()["slots"] == 3
            q = pinned(np.arange(0, 50_000, dtype=np.uint32))  # 13 jobs
            tk, out = srv.submit(q)
            srv.wait(tk)
            assert srv.stats()["jobs"] == 13
            assert np.array_equal(out, orc.point_search(keys, keys, q))


def test_learned_serving_needs_a_model(bt, cuda):
    keys = np.arange(1000, dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        with pytest.raises(bt.BTreeError):
            bt.Server(t, mode="learned")
