"""The CPU oracle, checked before it is trusted as ground truth.

* against numpy's searchsorted (an independent binary search);
* against known answers derived by hand from the reference's code;
* the literal restatement of the reference ("refc") against the ground truth, with
  the reference's documented divergences reproduced exactly.
The pin against the reference's own outputs is in test_golden_cpu.py.
"""
import numpy as np
import pytest

INV64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def np_point(keys, vals, q, miss):
    p = np.searchsorted(keys, q, side="left")
    pc = np.minimum(p, len(keys) - 1)
    hit = (p < len(keys)) & (keys[pc] == q)
    out = np.full(len(q), miss, dtype=vals.dtype)
    out[hit] = vals[pc[hit]]
    return out


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint32, np.uint64),
                                   (np.uint64, np.uint32), (np.uint64, np.uint64)])
def test_point_matches_searchsorted(orc, kt, vt):
    g = np.random.default_rng(7)
    hi = np.iinfo(kt).max
    keys = np.sort(g.integers(0, hi, size=20000, dtype=np.uint64, endpoint=True).astype(kt))
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    q = np.concatenate([keys[::3], g.integers(0, hi, size=5000, dtype=np.uint64).astype(kt),
                        np.array([0, hi], dtype=kt)])
    got = orc.point_search(keys, vals, q)
    exp = np_point(keys, vals, q, np.iinfo(vt).max)
    assert np.array_equal(got, exp)


def test_point_duplicates_first_occurrence(orc):
    keys = np.array([1, 3, 3, 3, 7, 7, 9], dtype=np.uint64)
    vals = np.arange(7, dtype=np.uint64) + 100
    q = np.array([3, 7, 9, 1, 2, 10, 0], dtype=np.uint64)
    got = orc.point_search(keys, vals, q)
    assert got.tolist() == [101, 104, 106, 100, int(INV64), int(INV64), int(INV64)]


def test_range_count_and_ids(orc):
    g = np.random.default_rng(3)
    keys = np.sort(g.integers(0, 1 << 20, size=30000, dtype=np.uint64).astype(np.uint32))
    vals = g.permutation(len(keys)).astype(np.uint32)
    lo = g.integers(0, 1 << 20, size=3000, dtype=np.uint64).astype(np.uint32)
    hi = (lo.astype(np.uint64) + g.integers(0, 4000, size=3000)).clip(0, (1 << 32) - 1).astype(np.uint32)
    hi[:10] = lo[:10] - 1  # some empty (lo > hi) ranges
    hi[:10] = np.where(lo[:10] == 0, 0, hi[:10])
    counts, offsets, ids = orc.range_search(keys, vals, lo, hi)
    l = np.searchsorted(keys, lo, "left")
    u = np.searchsorted(keys, hi, "right")
    exp = np.where(lo <= hi, u - l, 0)
    assert np.array_equal(counts, exp.astype(np.uint64))
    for i in range(0, 3000, 97):
        seg = ids[offsets[i]: offsets[i] + counts[i]]
        assert np.array_equal(seg, np.sort(vals[l[i]: l[i] + exp[i]]))


def test_rect_search_bruteforce(orc, wl):
    g = np.random.default_rng(11)
    x = g.integers(0, 512, size=4000).astype(np.uint16)
    y = g.integers(0, 512, size=4000).astype(np.uint16)
    z = wl.morton_u16(x, y)
    ids = np.arange(4000, dtype=np.uint32)
    o = np.lexsort((ids, z))
    zs, idss = z[o], ids[o]
    x0 = g.integers(0, 500, size=300).astype(np.uint16)
    y0 = g.integers(0, 500, size=300).astype(np.uint16)
    x1 = (x0 + g.integers(0, 64, size=300)).clip(0, 511).astype(np.uint16)
    y1 = (y0 + g.integers(0, 64, size=300)).clip(0, 511).astype(np.uint16)
    counts, offsets, got = orc.rect_search(zs, idss, x0, y0, x1, y1)
    for i in range(300):
        m = (x >= x0[i]) & (x <= x1[i]) & (y >= y0[i]) & (y <= y1[i])
        assert counts[i] == m.sum()
        assert np.array_equal(got[offsets[i]: offsets[i] + counts[i]], np.sort(ids[m]))


def test_morton_matches_bitwise(orc, wl):
    g = np.random.default_rng(5)
    x = g.integers(0, 1 << 16, size=200).astype(np.uint16)
    y = g.integers(0, 1 << 16, size=200).astype(np.uint16)
    z = wl.morton_u16(x, y)
    for i in range(200):
        assert orc.morton(x[i], y[i]) == z[i]
        # the reference's 64-bit interleave with interval 1 agrees on 16-bit inputs
        assert orc.zorder(x[i], y[i], 1, 1) == z[i]


# ---- the literal restatement of the reference ------------------------------

@pytest.mark.parametrize("n", [1, 7, 4999, 5000, 5001, 10000, 25001, 60000])
def test_refc_basic_equals_ground_truth(orc, n):
    """kernelSearchingNaiveOneStep == std::lower_bound exact match (unique keys)."""
    g = np.random.default_rng(n)
    keys = np.unique(g.integers(0, 1 << 40, size=n + 100, dtype=np.uint64))[:n]
    vals = np.arange(len(keys), dtype=np.uint64)
    t = orc.refc_build(keys, vals)
    q = np.concatenate([keys, keys + 1, [0, keys[-1] + 7]]).astype(np.uint64)
    assert np.array_equal(t.point_basic(q), orc.point_search(keys, vals, q))


def test_refc_grouped_needs_value_equals_key(orc):
    """Reference quirk: the grouped leaf search compares data[]
    (BPTreeExactSearch.cu:269-276): exact when value == key, wrong otherwise."""
    g = np.random.default_rng(2)
    keys = np.unique(g.integers(0, 1 << 32, size=60000, dtype=np.uint64))
    q = np.concatenate([keys[::2], g.integers(0, 1 << 32, size=2000, dtype=np.uint64)])
    t = orc.refc_build(keys, keys)
    assert np.array_equal(t.point_grouped(q), orc.point_search(keys, keys, q))
    ranks = np.arange(len(keys), dtype=np.uint64)
    t2 = orc.refc_build(keys, ranks)
    wrong = np.count_nonzero(t2.point_grouped(q) != orc.point_search(keys, ranks, q))
    assert wrong > len(q) // 4


def test_refc_range_known_answers(orc):
    """Hand-derived from BtreeRangeSearch.cu:297-374 on 2 full leaves of even
    keys 0, 2, ..., 19998 (data = key)."""
    keys = np.arange(0, 20000, 2, dtype=np.uint64)
    t = orc.refc_build(keys, keys)
    ep = t.range_endpoint(np.array([2, 10010, 9998, 10000], dtype=np.uint64))
    assert ep.tolist() == [(1 << 32) | 0, (5 << 32) | 1, (4999 << 32) | 0, (0 << 32) | 1]
    lo = np.array([2, 9990, 9998, 100], dtype=np.uint64)
    hi = np.array([4, 10010, 10000, 100], dtype=np.uint64)
    counts, rc = t.range_count(lo, hi)
    assert rc == 0
    # [2,4] in one leaf: the leaf position of 4 is 2, which equals the size
    # of the *parent* page (2 leaves), so BtreeRangeSearch.cu:284 rewrites it
    # to start-1 = 1 (the binary search broke with start = 2): 1 key counted.
    # [9990,10010]: the start-leaf loop stops at size-1 (drops 9998) and the
    # end-leaf loop stops before endPos (drops 10010): 11 keys, 9 counted.
    # [9998,10000]: both dropped: 0.
    assert counts.tolist() == [1, 9, 0, 1]
    exact = orc.range_count(keys, lo, hi)
    assert exact.tolist() == [2, 11, 2, 1]


def test_refc_range_count_undercounts(orc):
    """Across random ranges the reference's count is never above the exact
    count and is 0-3 low: the dropped last key of the start leaf, the dropped
    key at the end position, and the parent-size rewrite of a position."""
    g = np.random.default_rng(9)
    keys = np.unique(g.integers(0, 1 << 32, size=80000, dtype=np.uint64))
    keys = keys[: (len(keys) // 5000) * 5000]
    t = orc.refc_build(keys, keys)
    r = g.integers(0, len(keys), size=5000)
    w = g.integers(1, 20000, size=5000)
    lo = keys[r]
    hi = keys[np.minimum(r + w, len(keys) - 1)]
    ref, rc = t.range_count(lo, hi)
    assert rc == 0
    exact = orc.range_count(keys, lo, hi)
    d = exact.astype(np.int64) - ref.astype(np.int64)
    assert d.min() >= 0 and d.max() <= 3
    assert np.count_nonzero(d) > 0


def test_refc_buckets(orc):
    assert orc.bucket(0x1122334455667788, 0) == 0x11
    assert orc.bucket(0x1122334455667788, 7) == 0x88
    # 3-bit stride, 4-bit digit, product (grouping2d.cu:24-31)
    a, b = (0xF << 60), (0x3 << 60)
    assert orc.bucket2d(a, b, 1) == 0xF * 0x3
    assert orc.zorder_interval(0xFFFFFFFF) == 1
    assert orc.zorder_interval(1 << 33) == 2


def test_reference_query_families(wl):
    """The seeded restatements of the reference generator's query families."""
    import numpy as np
    mx = 10**9
    n = 200000
    u = wl.reference_queries("uniform", n, mx)
    assert u.max() <= mx and abs(u.mean() / mx - 0.5) < 0.01
    for kind, sig in (("normal", 0.35), ("normal_wide", 0.63)):
        x = wl.reference_queries(kind, n, mx).astype(np.float64)
        assert x.min() >= 0 and x.max() <= mx
        inside = x[x != mx // 2]
        assert abs(np.median(x) / (mx / 2) - 1) < 0.02
        assert abs(inside.std() / (sig * mx / 2) - 1) < (0.05 if kind == "normal" else 0.5)
    z = wl.reference_queries("zipf", n, mx)
    assert z.min() >= 1 and (z == 1).mean() > 0.03  # rank 1 is the most frequent
    mg = wl.reference_queries("multi_gaussian", n, mx)
    assert len(np.unique(mg)) <= 10  # five clusters of nearly one value each
    assert np.array_equal(wl.reference_queries("zipf", 1000, mx), wl.reference_queries("zipf", 1000, mx))


def _line_fits(xs, ys, eps):
    """Is there a line within eps of every point?  (LP feasibility)"""
    from scipy.optimize import linprog
    x = (xs - xs[0]).astype(np.float64)
    y = ys.astype(np.float64)
    a = np.vstack([np.c_[x, np.ones_like(x)], np.c_[-x, -np.ones_like(x)]])
    b = np.r_[y + eps, eps - y]
    r = linprog([0, 0], A_ub=a, b_ub=b, bounds=[(None, None), (None, None)], method="highs")
    return r.status == 0


@pytest.mark.parametrize("eps", [1, 4, 16])
def test_pla_segments_are_feasible_and_maximal(orc, eps):
    """Every segment of the oracle's error-bounded segmentation admits a line
    within eps of its points, and none could take one more point."""
    g = np.random.default_rng(eps)
    keys = np.cumsum(np.floor(g.lognormal(4.0, 2.0, size=2500)).astype(np.uint64) + 1)
    st, sl, ic = orc.pla_segments(keys, eps)
    bounds = list(st.astype(np.int64)) + [len(keys)]
    for s, e, slope, icpt in zip(bounds[:-1], bounds[1:], sl, ic):
        r = np.arange(e - s, dtype=np.float64)
        assert _line_fits(keys[s:e], r, eps)
        # the line the oracle reports is itself within eps (float64 rounding aside)
        pred = icpt + slope * (keys[s:e] - keys[s]).astype(np.float64)
        assert np.max(np.abs(pred - r)) <= eps + 1e-6
        if e < len(keys):
            assert not _line_fits(keys[s:e + 1], np.arange(e + 1 - s, dtype=np.float64), eps)


def test_pla_segment_counts_shrink_with_eps(orc):
    keys = np.cumsum(np.floor(np.random.default_rng(2).lognormal(4.0, 2.0, size=1 << 18))
                     .astype(np.uint64) + 1)
    counts = [orc.pla_segments(keys, e, lines=False) for e in (8, 16, 64, 256)]
    assert counts == sorted(counts, reverse=True) and counts[-1] < counts[0]
    # chunking adds at most one segment per chunk boundary
    full = orc.pla_segments(keys, 64, lines=False)
    chunked = orc.pla_segments(keys, 64, chunk=1 << 14, lines=False)
    assert full <= chunked <= full + (len(keys) >> 14)
