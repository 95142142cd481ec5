"""Batched forest: many uneven trees built and searched in one graph launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def make_forest(g, sizes, kt):
    keys, off = [], [0]
    for n in sizes:
        k = np.unique(g.integers(0, np.iinfo(kt).max, size=n + n // 4 + 4, dtype=np.uint64))[:n]
        keys.append(k.astype(kt))
        off.append(off[-1] + len(keys[-1]))
    return keys, np.array(off, dtype=np.uint64)


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint64, np.uint64),
                                   (np.uint32, np.uint64)])
@pytest.mark.parametrize("cfg,tile", [((4, 1), 1024), ((8, 2), 256), ((2, 1), 32), ((8, 1), 4096)])
def test_forest_matches_oracle(bt, orc, cuda, kt, vt, cfg, tile):
    import torch
    g = np.random.default_rng(7)
    sizes = [0, 1, 7, 8, 9, 100, 1000, 5000, 0, 33333, 2, 70001, 1 << 16, 3]
    keys, off = make_forest(g, sizes, kt)
    vals = [np.arange(len(k), dtype=vt) * 3 + 1 for k in keys]
    qs, qoff, los, his, roff = [], [0], [], [], [0]
    for k in keys:
        m = int(g.integers(0, 3000))
        q = g.integers(0, np.iinfo(kt).max, size=m, dtype=np.uint64).astype(kt)
        if len(k):
            q[: m * 4 // 5] = k[g.integers(0, len(k), size=m * 4 // 5)]
        qs.append(q)
        qoff.append(qoff[-1] + m)
        r = int(g.integers(0, 50))
        if len(k):
            a = g.integers(0, len(k), size=r)
            w = g.integers(1, 1 << 12, size=r)
            lo, hi = k[a], k[np.minimum(a + w - 1, len(k) - 1)]
        else:
            lo = g.integers(0, 1000, size=r).astype(kt)
            hi = lo + 5
        los.append(lo.astype(kt))
        his.append(hi.astype(kt))
        roff.append(roff[-1] + r)
    cat = lambda xs, t: np.concatenate(xs).astype(t) if len(xs) else np.zeros(0, t)  # noqa: E731
    dq = dev(cat(qs, kt), cuda)
    dlo, dhi = dev(cat(los, kt), cuda), dev(cat(his, kt), cuda)
    out = torch.empty(len(dq), dtype={4: torch.uint32, 8: torch.uint64}[np.dtype(vt).itemsize],
                      device=cuda)
    counts = torch.empty(len(dlo), dtype=torch.uint64, device=cuda)
    with bt.Forest(dev(cat(keys, kt), cuda), dev(cat(vals, vt), cuda), off) as f:
        with f.plan(dq, qoff, out, dlo, dhi, roff, counts, *cfg, tile=tile) as p:
            for _ in range(2):  # the graph replays
                out.fill_(0)
                counts.fill_(7)
                p.run()
                torch.cuda.synchronize()
                got, gotc = out.cpu().numpy(), counts.cpu().numpy()
                for t, k in enumerate(keys):
                    sl = slice(int(qoff[t]), int(qoff[t + 1]))
                    exp = orc.point_search(k, vals[t], qs[t]) if len(k) else \
                        np.full(len(qs[t]), np.iinfo(vt).max, dtype=vt)
                    assert np.array_equal(got[sl], exp), t
                    rs = slice(int(roff[t]), int(roff[t + 1]))
                    expc = orc.range_count(k, los[t], his[t]) if len(k) else np.zeros(len(los[t]))
                    assert np.array_equal(gotc[rs], expc), t


def test_forest_rejects_unsorted_tree(bt, cuda):
    keys = np.array([1, 2, 3, 9, 5, 6], dtype=np.uint32)
    with pytest.raises(bt.BTreeError) as e:
        bt.Forest(dev(keys, cuda), dev(keys, cuda), np.array([0, 3, 6], dtype=np.uint64))
    assert e.value.name == "BT_ERR_UNSORTED"
