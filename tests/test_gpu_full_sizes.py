"""The benchmark workloads at their full sizes.

Exactness against the oracle is checked on a sample where the oracle would
take too long on the whole batch; the whole batch is checked through
properties that hold at any size: results do not depend on the search mode
or the search shape, a found value is the rank of a key equal to the query
(value = rank), a query drawn from the keys is always found, range counts
over unique keys are rank differences, and rectangle answers are sorted,
inside their box, and as many as their count.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MISS32 = np.uint32(0xFFFFFFFF)


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def test_plain_point_search_2e20(bt, orc, wl, cuda):
    """2^20 uniform u32 keys, 2^20 queries (half existing keys), basic search:
    the whole batch against the oracle."""
    keys, vals, q = wl.point_uniform(1 << 20, 1 << 20)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        got = t.point_search(dev(q, cuda), mode="basic").cpu().numpy()
    assert np.array_equal(got, exp)
    assert np.all(got[0::2] != MISS32)  # every query drawn from the keys is found


def test_grouped_point_search_2e26_keys_2e24_zipf(bt, orc, wl, cuda):
    """2^26 keys, 2^24 Zipf queries: grouped == basic on the whole batch, the
    whole batch against the oracle, and the value = rank property."""
    keys, vals, q = wl.point_zipf()
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        dq = dev(q, cuda)
        basic = t.point_search(dq, mode="basic").cpu().numpy()
        grouped = t.point_search(dq, mode="grouped").cpu().numpy()
    assert np.array_equal(basic, exp)
    assert np.array_equal(grouped, exp)
    found = grouped != MISS32
    assert np.array_equal(keys[grouped[found].astype(np.int64)], q[found])


def test_rectangles_2e24_points_2e20_boxes(bt, orc, wl, cuda):
    """2^24 points, 2^20 boxes: the first 8192 boxes against the oracle; for
    every box, IDs strictly ascending, inside the box, and `count` of them."""
    z, ids, x0, y0, x1, y1 = wl.zorder_points()
    with bt.Tree.build(dev(z, cuda), dev(ids, cuda)) as t:
        c, off, got = bt.rect_search(t, *(dev(a, cuda) for a in (x0, y0, x1, y1)))
    c, off, got = c.cpu().numpy(), off.cpu().numpy(), got.cpu().numpy()
    s = slice(0, 8192)
    ec, _, ei = orc.rect_search(z, ids, x0[s], y0[s], x1[s], y1[s])
    assert np.array_equal(c[s], ec)
    assert np.array_equal(got[: int(off[8191] + c[8191])], ei)
    assert int(c.sum()) == len(got)
    assert np.array_equal(off[1:], np.cumsum(c)[:-1])
    # every hit inside its box, IDs ascending within each box
    box = np.repeat(np.arange(len(c)), c.astype(np.int64))
    zid = np.empty(len(z), dtype=np.uint32)
    zid[ids] = z
    hz = zid[got]
    hx, hy = wl.compact_u16(hz), wl.compact_u16(hz >> np.uint32(1))
    assert np.all((hx >= x0[box]) & (hx <= x1[box]) & (hy >= y0[box]) & (hy <= y1[box]))
    d = np.diff(got.astype(np.int64))
    same = box[1:] == box[:-1]
    assert np.all(d[same] > 0)


def test_forest_4096_trees(bt, orc, wl, cuda):
    """4,096 trees (620 M keys), one plan launch: found values point back at
    their query, queries that are keys of their tree are found, range counts
    are rank differences; every 64th tree against the oracle."""
    import torch
    keys, vals, koff, q, qoff, lo, hi, roff = wl.forest()
    with bt.Forest(dev(keys, cuda), dev(vals, cuda), koff) as f:
        out = torch.empty(len(q), dtype=torch.uint32, device=cuda)
        counts = torch.empty(len(lo), dtype=torch.uint64, device=cuda)
        dq, dlo, dhi = dev(q, cuda), dev(lo, cuda), dev(hi, cuda)
        with f.plan(dq, qoff, out, dlo, dhi, roff, counts, 4, 1, tile=512) as p:
            p.run()
            torch.cuda.synchronize()
        res, cnt = out.cpu().numpy(), counts.cpu().numpy()
    sizes = np.diff(koff.astype(np.int64))
    tq = np.repeat(np.arange(len(sizes)), np.diff(qoff.astype(np.int64)))
    found = res != MISS32
    assert np.array_equal(keys[koff[tq[found]].astype(np.int64) + res[found]], q[found])
    tr = np.repeat(np.arange(len(sizes)), np.diff(roff.astype(np.int64)))
    for t in range(0, len(sizes), 64):
        k = keys[koff[t]:koff[t + 1]]
        v = vals[koff[t]:koff[t + 1]]
        qs = slice(int(qoff[t]), int(qoff[t + 1]))
        rs = slice(int(roff[t]), int(roff[t + 1]))
        assert np.array_equal(res[qs], orc.point_search(k, v, q[qs]))
        assert np.array_equal(cnt[rs], orc.range_count(k, lo[rs], hi[rs]))
        assert np.all(tr[rs] == t)


def test_learned_index_2e28_lognormal(bt, orc, wl, cuda):
    """2^28 u64 keys from lognormal gaps, 2^24 queries: the learned search
    equals the plain search on the whole batch; 2^20 of them against the
    oracle."""
    keys = wl.lognormal_keys()
    vals = np.arange(len(keys), dtype=np.uint64)
    g = np.random.default_rng(11)
    nq = 1 << 24
    q = keys[g.integers(0, len(keys), size=nq)]
    m = g.random(nq) < 0.10
    q[m] = g.integers(int(keys[0]), int(keys[-1]) + 1, size=int(m.sum()), dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        dq = dev(q, cuda)
        plain = t.point_search(dq, mode="basic").cpu().numpy()
        t.learned_train()
        learned = t.point_search_learned(dq).cpu().numpy()
    assert np.array_equal(learned, plain)
    s = slice(0, 1 << 20)
    assert np.array_equal(plain[s], orc.point_search(keys, vals, q[s]))
    assert np.all(plain[~m] != np.uint64(0xFFFFFFFFFFFFFFFF))
