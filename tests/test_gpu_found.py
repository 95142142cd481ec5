"""Found flags (bt_point_search_found): a stored value of all-ones is told
apart from a miss, in every point-search mode, against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TYPES = [(np.uint32, np.uint32), (np.uint32, np.uint64), (np.uint64, np.uint32),
         (np.uint64, np.uint64)]


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def case(kt, vt, n, nq, seed):
    g = np.random.default_rng(seed)
    hi = int(np.iinfo(kt).max)
    keys = np.unique(g.integers(0, hi, size=n + n // 8 + 16, dtype=np.uint64,
                                endpoint=True))[:n].astype(kt)
    keys[-1] = hi  # the all-ones key is a key too
    keys = np.unique(keys)
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    vals[::7] = np.iinfo(vt).max  # stored values equal to the miss marker
    q = np.concatenate([keys[g.integers(0, len(keys), size=nq // 2)],
                        g.integers(0, hi, size=nq - nq // 2, dtype=np.uint64,
                                   endpoint=True).astype(kt)])
    g.shuffle(q)
    return keys, vals, q


@pytest.mark.parametrize("kt,vt", TYPES)
@pytest.mark.parametrize("mode", ["basic", "grouped", "learned"])
def test_found_flags_match_the_oracle(bt, orc, cuda, kt, vt, mode):
    keys, vals, q = case(kt, vt, 300007, 100000, 5)
    exp = orc.point_search(keys, vals, q)
    inside = np.isin(q, keys)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        if mode == "learned":
            t.learned_train(max_error=32, iterations=50)
        out, found = t.point_search_found(dev(q, cuda), mode=mode)
        out, found = out.cpu().numpy(), found.cpu().numpy()
        assert np.array_equal(out, exp)
        assert np.array_equal(found.astype(bool), inside)
        # hits whose stored value is all-ones look like misses by value alone
        assert np.count_nonzero(inside & (out == np.iinfo(vt).max)) > 0
        # the values agree with the call without flags
        assert np.array_equal(t.point_search(dev(q, cuda), mode=mode).cpu().numpy(), out)


def test_found_flags_grouped_window_path(bt, orc, cuda):
    """2^21 queries and more take the per-group window kernel."""
    keys, vals, q = case(np.uint32, np.uint32, 1 << 20, (1 << 21) + 5, 9)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        out, found = t.point_search_found(dev(q, cuda), mode="grouped")
        assert np.array_equal(out.cpu().numpy(), orc.point_search(keys, vals, q))
        assert np.array_equal(found.cpu().numpy().astype(bool), np.isin(q, keys))


def test_found_flags_empty_tree_and_bad_arguments(bt, cuda):
    import ctypes
    import torch
    empty = np.zeros(0, dtype=np.uint64)
    q = np.arange(10, dtype=np.uint64)
    with bt.Tree.build(dev(empty, cuda), dev(empty, cuda)) as t:
        out, found = t.point_search_found(dev(q, cuda))
        assert (out.cpu().numpy() == np.iinfo(np.uint64).max).all()
        assert (found.cpu().numpy() == 0).all()
    keys = np.arange(100, dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        dq = dev(q, cuda)
        out = torch.empty(10, dtype=torch.uint64, device=cuda)
        st = bt.lib().bt_point_search_found(t.handle, 0, ctypes.c_void_p(dq.data_ptr()), 10,
                                            ctypes.c_void_p(out.data_ptr()), None, None)
        assert st != 0  # no found array
