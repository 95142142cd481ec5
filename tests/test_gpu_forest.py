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


def forest_case(kt, vt, cuda, seed=7):
    """Uneven trees (some empty) with point queries (80% hits) and ranges."""
    import torch
    g = np.random.default_rng(seed)
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
    c = dict(keys=keys, vals=vals, off=off, qs=qs, qoff=qoff, los=los, his=his, roff=roff)
    c["dkeys"], c["dvals"] = dev(cat(keys, kt), cuda), dev(cat(vals, vt), cuda)
    c["dq"] = dev(cat(qs, kt), cuda)
    c["dlo"], c["dhi"] = dev(cat(los, kt), cuda), dev(cat(his, kt), cuda)
    c["out"] = torch.empty(len(c["dq"]), dtype={4: torch.uint32, 8: torch.uint64}[np.dtype(vt).itemsize],
                           device=cuda)
    c["counts"] = torch.empty(len(c["dlo"]), dtype=torch.uint64, device=cuda)
    return c


def check_forest(orc, c, vt):
    got, gotc = c["out"].cpu().numpy(), c["counts"].cpu().numpy()
    for t, k in enumerate(c["keys"]):
        sl = slice(int(c["qoff"][t]), int(c["qoff"][t + 1]))
        exp = orc.point_search(k, c["vals"][t], c["qs"][t]) if len(k) else \
            np.full(len(c["qs"][t]), np.iinfo(vt).max, dtype=vt)
        assert np.array_equal(got[sl], exp), t
        rs = slice(int(c["roff"][t]), int(c["roff"][t + 1]))
        expc = orc.range_count(k, c["los"][t], c["his"][t]) if len(k) else np.zeros(len(c["los"][t]))
        assert np.array_equal(gotc[rs], expc), t


def run_plan(f, c, cfg, tile):
    import torch
    with f.plan(c["dq"], c["qoff"], c["out"], c["dlo"], c["dhi"], c["roff"], c["counts"], *cfg,
                tile=tile) as p:
        c["out"].fill_(0)
        c["counts"].fill_(7)
        p.run()
        torch.cuda.synchronize()


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint64, np.uint64),
                                   (np.uint32, np.uint64)])
@pytest.mark.parametrize("cfg,tile", [((4, 1), 1024), ((8, 2), 256), ((2, 1), 32), ((8, 1), 4096)])
def test_forest_matches_oracle(bt, orc, cuda, kt, vt, cfg, tile):
    import torch
    c = forest_case(kt, vt, cuda)
    with bt.Forest(c["dkeys"], c["dvals"], c["off"]) as f:
        with f.plan(c["dq"], c["qoff"], c["out"], c["dlo"], c["dhi"], c["roff"], c["counts"], *cfg,
                    tile=tile) as p:
            for _ in range(2):  # the graph replays
                c["out"].fill_(0)
                c["counts"].fill_(7)
                p.run()
                torch.cuda.synchronize()
                check_forest(orc, c, vt)


@pytest.mark.parametrize("fanout", [1, 4, 64, 4096])
def test_forest_stage_fanout(bt, orc, cuda, fanout):
    """The staged-root fanout changes which level a work item stages, never
    the answers."""
    c = forest_case(np.uint64, np.uint32, cuda, seed=11)
    with bt.Forest(c["dkeys"], c["dvals"], c["off"]) as f:
        f.set_stage_fanout(fanout)
        run_plan(f, c, (4, 1), 512)
        check_forest(orc, c, np.uint32)


def test_forest_tuner_picks_fanout_and_caches(bt, orc, cuda, tmp_path):
    import importlib
    at = importlib.import_module("b-tree-index-searching_b200.autotune")
    c = forest_case(np.uint32, np.uint32, cuda, seed=3)
    cache = str(tmp_path / "forest.json")
    with bt.Forest(c["dkeys"], c["dvals"], c["off"]) as f:
        args = (f, c["dq"], c["qoff"], c["out"], c["dlo"], c["dhi"], c["roff"], c["counts"])
        lanes, rounds, tile, fanout, ms = at.tune_forest(*args, repeats=1, cache_path=cache)
        assert fanout in at.FOREST_FANOUTS and (lanes, rounds) in at.FOREST_SHAPES
        assert len(ms) == len(at.FOREST_SHAPES) * len(at.FOREST_TILES) + len(at.FOREST_FANOUTS) - 1
        assert at.tune_forest(*args, repeats=1, cache_path=cache)[:4] == (lanes, rounds, tile, fanout)
        run_plan(f, c, (lanes, rounds), tile)
        check_forest(orc, c, np.uint32)
    with bt.Forest(c["dkeys"], c["dvals"], c["off"]) as f:
        with pytest.raises(bt.BTreeError):
            f.set_stage_fanout(0)


def test_forest_rejects_unsorted_tree(bt, cuda):
    keys = np.array([1, 2, 3, 9, 5, 6], dtype=np.uint32)
    with pytest.raises(bt.BTreeError) as e:
        bt.Forest(dev(keys, cuda), dev(keys, cuda), np.array([0, 3, 6], dtype=np.uint64))
    assert e.value.name == "BT_ERR_UNSORTED"
