"""Device sort of unsorted (key, value) input and the build from it, against
numpy's stable sort and the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint32, np.uint64),
                                   (np.uint64, np.uint32), (np.uint64, np.uint64)])
@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 100003, 1 << 21])
def test_sort_pairs_is_a_stable_sort(bt, cuda, kt, vt, n):
    g = np.random.default_rng(n + np.dtype(kt).itemsize * 3 + np.dtype(vt).itemsize)
    hi = int(np.iinfo(kt).max)
    keys = g.integers(0, hi, size=n, dtype=np.uint64, endpoint=True).astype(kt)
    keys[: n // 3] = keys[n // 3: 2 * (n // 3)]  # duplicates
    keys[:1] = hi
    vals = np.arange(n, dtype=vt)  # input order, to check stability
    ok, ov = bt.sort_pairs(dev(keys, cuda), dev(vals, cuda))
    o = np.argsort(keys, kind="stable")
    assert np.array_equal(ok.cpu().numpy(), keys[o])
    assert np.array_equal(ov.cpu().numpy(), vals[o])


@pytest.mark.parametrize("kt", [np.uint32, np.uint64])
def test_build_unsorted_searches_like_the_sorted_build(bt, orc, cuda, kt):
    g = np.random.default_rng(9)
    n = 300001
    keys = np.unique(g.integers(0, int(np.iinfo(kt).max), size=n, dtype=np.uint64)).astype(kt)
    vals = g.integers(0, 1 << 31, size=len(keys), dtype=np.uint64).astype(np.uint32)
    p = g.permutation(len(keys))
    q = np.concatenate([keys[g.integers(0, len(keys), size=50000)],
                        g.integers(0, int(np.iinfo(kt).max), size=50000, dtype=np.uint64).astype(kt)])
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build_unsorted(dev(keys[p], cuda), dev(vals[p], cuda)) as t:
        assert t.info.num_keys == len(keys)
        for mode in ("basic", "grouped"):
            assert np.array_equal(t.point_search(dev(q, cuda), mode=mode).cpu().numpy(), exp)


def test_sort_rejects_aliased_outputs(bt, cuda):
    import ctypes
    import torch
    k = torch.zeros(10, dtype=torch.int32, device=cuda)
    P = ctypes.c_void_p
    st = bt.lib().bt_sort_pairs(P(k.data_ptr()), P(k.data_ptr()), 10, 4, 4, P(k.data_ptr()),
                                P(k.data_ptr()), None)
    assert st == 1
