"""Range search on the GPU against the CPU oracle (counts + sorted hit IDs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = ("basic", "2d", "zorder")


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def ranges(keys, kt, g, nq):
    hi_v = int(np.iinfo(kt).max)
    lo = g.integers(0, hi_v, size=nq, dtype=np.uint64, endpoint=True)
    span = min(hi_v // max(1, len(keys)) * 64, 1 << 62)
    w = g.integers(0, max(2, span), size=nq, dtype=np.uint64)
    hi = lo + np.minimum(w, np.uint64(hi_v) - lo)  # no wrap-around
    # exact key endpoints, single-key ranges, empty (lo > hi) and full ranges
    k = keys.astype(np.uint64)
    m = nq // 8
    idx = g.integers(0, len(keys), size=m)
    lo[:m] = k[idx]
    hi[:m] = k[np.minimum(idx + g.integers(0, 40, size=m), len(keys) - 1)]
    lo[m:2 * m] = k[idx]
    hi[m:2 * m] = k[idx]
    lo[2 * m:2 * m + 16] = 5
    hi[2 * m:2 * m + 16] = 4
    lo[-1], hi[-1] = 0, hi_v
    return lo.astype(kt), hi.astype(kt)


@pytest.mark.parametrize("kt", [np.uint32, np.uint64])
@pytest.mark.parametrize("n", [1, 5, 8, 33, 1000, 5000, 5001, 70001, 1 << 18])
@pytest.mark.parametrize("mode", MODES)
def test_range_count(bt, orc, cuda, kt, n, mode):
    g = np.random.default_rng(n + np.dtype(kt).itemsize)
    keys = np.unique(g.integers(0, np.iinfo(kt).max, size=n + 64, dtype=np.uint64))[:n].astype(kt)
    vals = np.arange(len(keys), dtype=np.uint32)
    lo, hi = ranges(keys, kt, g, 20000)
    exp = orc.range_count(keys, lo, hi)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        got = t.range_count(dev(lo, cuda), dev(hi, cuda), mode=mode).cpu().numpy()
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("vt", [np.uint32, np.uint64])
@pytest.mark.parametrize("sorted_vals", [True, False])
@pytest.mark.parametrize("mode", MODES)
def test_range_ids(bt, orc, cuda, vt, sorted_vals, mode):
    g = np.random.default_rng(21 + int(sorted_vals))
    keys = np.unique(g.integers(0, 1 << 32, size=300000, dtype=np.uint64)).astype(np.uint32)
    vals = np.arange(len(keys), dtype=vt)
    if not sorted_vals:
        vals = g.permutation(vals).astype(vt)
    lo, hi = ranges(keys, np.uint32, g, 30000)
    # keep the widest ranges under the 4096-hit cap of the unsorted-value path
    hi = np.where(lo.astype(np.uint64) + (1 << 24) < hi, lo + (1 << 24), hi).astype(np.uint32)
    ec, eo, ei = orc.range_search(keys, vals, lo, hi)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        assert bool(t.info.values_sorted) == sorted_vals
        c, o, ids = t.range_search(dev(lo, cuda), dev(hi, cuda), mode=mode)
    assert np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(o.cpu().numpy(), eo)
    assert np.array_equal(ids.cpu().numpy(), ei)


def test_range_capacity_error(bt, cuda):
    import ctypes
    import torch
    keys = np.arange(0, 1000, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        lo = dev(np.array([0, 10], dtype=np.uint32), cuda)
        hi = dev(np.array([99, 19], dtype=np.uint32), cuda)
        counts = torch.empty(2, dtype=torch.uint64, device=cuda)
        offs = torch.empty(2, dtype=torch.uint64, device=cuda)
        ids = torch.empty(50, dtype=torch.uint32, device=cuda)
        total = ctypes.c_uint64()
        st = bt.lib().bt_range_search(t.handle, 0, ctypes.c_void_p(lo.data_ptr()),
                                      ctypes.c_void_p(hi.data_ptr()), 2,
                                      ctypes.c_void_p(counts.data_ptr()),
                                      ctypes.c_void_p(offs.data_ptr()),
                                      ctypes.c_void_p(ids.data_ptr()), 50, ctypes.byref(total),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 5 and total.value == 110
        assert counts.cpu().numpy().tolist() == [100, 10]
        assert offs.cpu().numpy().tolist() == [0, 100]


def test_range_host_pipeline(bt, orc, cuda):
    g = np.random.default_rng(8)
    keys = np.unique(g.integers(0, 1 << 32, size=1 << 20, dtype=np.uint64)).astype(np.uint32)
    lo, hi = ranges(keys, np.uint32, g, (1 << 21) + 7)
    exp = orc.range_count(keys, lo, hi)
    with bt.Tree.build(keys, keys) as t:
        for mode in MODES:
            assert np.array_equal(t.range_count(lo, hi, mode=mode), exp), mode


def test_range_ids_long_unsorted_segments(bt, orc, cuda):
    """Result sets longer than the shared-memory sort (4096 values) whose
    values do not ascend with the keys."""
    g = np.random.default_rng(33)
    keys = np.unique(g.integers(0, 1 << 32, size=200000, dtype=np.uint64)).astype(np.uint32)
    vals = g.permutation(len(keys)).astype(np.uint32)
    lo = np.array([0, keys[10], keys[5000], 7], dtype=np.uint32)
    hi = np.array([0xFFFFFFFF, keys[9000], keys[5100], 9], dtype=np.uint32)
    ec, eo, ei = orc.range_search(keys, vals, lo, hi)
    assert ec.max() > 4096
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        c, o, ids = t.range_search(dev(lo, cuda), dev(hi, cuda))
    assert np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(ids.cpu().numpy(), ei)


@pytest.mark.parametrize("nr,wmin,width", [(5000, 1, 40), (3000, 1, 200), (2000, 1, 1500),
                                           (70000, 257, 300)])
def test_range_ids_unsorted_segment_tiers(bt, orc, cuda, nr, wmin, width):
    """Unsorted values in every segment-sort tier: warp ranking (<= 256
    values, with duplicate values), one CTA per listed segment (<= 4096), and
    more medium segments than the list holds (70000 x ~300 values)."""
    g = np.random.default_rng(nr + width)
    keys = np.unique(g.integers(0, 1 << 32, size=1 << 20, dtype=np.uint64)).astype(np.uint32)
    vals = g.permutation(len(keys)).astype(np.uint32)
    m = len(vals[1::7])
    vals[0:7 * m:7] = vals[1::7]  # duplicate values
    r = g.integers(0, len(keys) - width, size=nr)
    w = g.integers(wmin, width + 1, size=nr)
    lo, hi = keys[r], keys[r + w - 1]
    ec, eo, ei = orc.range_search(keys, vals, lo, hi)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        c, o, ids = t.range_search(dev(lo, cuda), dev(hi, cuda))
    assert np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(o.cpu().numpy(), eo)
    assert np.array_equal(ids.cpu().numpy(), ei)
