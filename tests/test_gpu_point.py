"""Point search on the GPU against the CPU oracle (bit-exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TYPES = [(np.uint32, np.uint32), (np.uint32, np.uint64), (np.uint64, np.uint32),
         (np.uint64, np.uint64)]
SIZES = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 127, 128, 129, 255, 256, 257, 511,
         512, 513, 1023, 1024, 1025, 4095, 4096, 4097, 5000, 5001, 8191, 8193, 32768, 33333,
         65537, 200003]


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def make_keys(n, kt, g, dense_ends=True):
    hi = int(np.iinfo(kt).max)
    k = np.unique(g.integers(0, hi, size=n + n // 8 + 16, dtype=np.uint64, endpoint=True))
    k = k[:n].astype(kt)
    if dense_ends and n >= 4:
        k[0] = 0
        k[-1] = np.iinfo(kt).max
        k = np.unique(k)
    return k


def queries_for(keys, kt, g, extra=4096):
    hi = int(np.iinfo(kt).max)
    k64 = keys.astype(np.uint64)
    parts = [keys, (k64 + 1).astype(kt), (k64 - 1).astype(kt),
             g.integers(0, hi, size=extra, dtype=np.uint64, endpoint=True).astype(kt),
             np.array([0, 1, hi, hi - 1], dtype=kt)]
    q = np.concatenate(parts)
    g.shuffle(q)
    return q


@pytest.mark.parametrize("kt,vt", TYPES)
@pytest.mark.parametrize("n", SIZES)
def test_point_exact(bt, orc, cuda, kt, vt, n):
    g = np.random.default_rng(n * 7 + np.dtype(kt).itemsize + 3 * np.dtype(vt).itemsize)
    keys = make_keys(n, kt, g)
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    q = queries_for(keys, kt, g)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        assert t.info.num_keys == len(keys)
        for mode in ("basic", "grouped"):
            got = t.point_search(dev(q, cuda), mode=mode).cpu().numpy()
            assert np.array_equal(got, exp), mode


@pytest.mark.parametrize("kt", [np.uint32, np.uint64])
def test_point_duplicates(bt, orc, cuda, kt):
    g = np.random.default_rng(4)
    keys = np.sort(g.integers(0, 3000, size=50000).astype(kt))  # heavy duplicates
    vals = np.arange(len(keys), dtype=np.uint64)
    q = np.arange(0, 3100, dtype=kt)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        for mode in ("basic", "grouped"):
            assert np.array_equal(t.point_search(dev(q, cuda), mode=mode).cpu().numpy(), exp)


def test_point_host_pipeline(bt, orc, cuda):
    """Host buffers, several pipelined chunks."""
    g = np.random.default_rng(12)
    keys = make_keys(1 << 20, np.uint32, g, dense_ends=False)
    vals = np.arange(len(keys), dtype=np.uint32)
    q = g.integers(0, 1 << 32, size=(1 << 22) + 12345, dtype=np.uint64).astype(np.uint32)
    q[::2] = keys[g.integers(0, len(keys), size=len(q[::2]))]
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(keys, vals) as t:  # host build
        for mode in ("basic", "grouped"):
            assert np.array_equal(t.point_search(q, mode=mode), exp), mode


def test_empty_tree_and_empty_batch(bt, cuda):
    import torch
    keys = np.zeros(0, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        q = dev(np.array([0, 5, 0xFFFFFFFF], dtype=np.uint32), cuda)
        assert t.point_search(q).cpu().numpy().tolist() == [0xFFFFFFFF] * 3
        lo = dev(np.array([0], dtype=np.uint32), cuda)
        assert t.range_count(lo, lo).cpu().numpy().tolist() == [0]
    keys = np.arange(10, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        e = torch.empty(0, dtype=torch.uint32, device=cuda)
        assert t.point_search(e).numel() == 0


def test_unsorted_build_rejected(bt, cuda):
    keys = np.array([1, 5, 3, 9], dtype=np.uint32)
    with pytest.raises(bt.BTreeError) as ei:
        bt.Tree.build(dev(keys, cuda), dev(keys, cuda))
    assert ei.value.name == "BT_ERR_UNSORTED"


def test_grouping_is_a_stable_permutation(bt, cuda):
    g = np.random.default_rng(6)
    keys = make_keys(100000, np.uint32, g, dense_ends=False)
    q = g.integers(0, 1 << 32, size=300001, dtype=np.uint64).astype(np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        gq, perm = t.group(dev(q, cuda))
        gq, perm = gq.cpu().numpy(), perm.cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(perm), np.arange(len(q)))
    assert np.array_equal(gq, q[perm])
    shift = max(0, int(keys[-1]).bit_length() - 8)
    d = np.minimum(gq.astype(np.uint64) >> np.uint64(shift), 255)
    assert np.all(np.diff(d.astype(np.int64)) >= 0)          # grouped by digit
    same = np.diff(d.astype(np.int64)) == 0
    assert np.all(np.diff(perm)[same] > 0)                  # stable inside a group


@pytest.mark.parametrize("kt,vt", TYPES)
@pytest.mark.parametrize("cfg", [(8, 1), (8, 2), (4, 1), (4, 2), (2, 1)])
def test_every_search_config(bt, orc, cuda, kt, vt, cfg):
    """Results do not depend on the kernel shape the autotuner picks."""
    g = np.random.default_rng(31)
    keys = make_keys(70001, kt, g)
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    q = queries_for(keys, kt, g, extra=20000)
    lo = np.minimum(q, np.roll(q, 1))
    hi = np.maximum(q, np.roll(q, 1))
    exp = orc.point_search(keys, vals, q)
    expc = orc.range_count(keys, lo, hi)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        t.set_search_config(*cfg)
        assert (t.info.lanes_per_query, t.info.rounds) == cfg
        for mode in ("basic", "grouped"):
            assert np.array_equal(t.point_search(dev(q, cuda), mode=mode).cpu().numpy(), exp)
        for mode in ("basic", "2d", "zorder"):
            got = t.range_count(dev(lo, cuda), dev(hi, cuda), mode=mode).cpu().numpy()
            assert np.array_equal(got, expc)


def test_autotuner_picks_a_supported_config(bt, orc, cuda):
    import importlib
    at = importlib.import_module("b-tree-index-searching_b200.autotune")
    g = np.random.default_rng(5)
    keys = make_keys(1 << 18, np.uint32, g, dense_ends=False)
    q = g.integers(0, 1 << 32, size=1 << 18, dtype=np.uint64).astype(np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        lanes, slots, ms = at.tune(t, dev(q, cuda), mode="basic", repeats=2)
        assert (lanes, slots) in bt.Tree.SEARCH_CONFIGS and len(ms) == 5
        got = t.point_search(dev(q, cuda)).cpu().numpy()
    assert np.array_equal(got, orc.point_search(keys, keys, q))


def test_wrong_query_width_rejected(bt, cuda):
    keys = np.arange(100, dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        with pytest.raises(ValueError):
            t.point_search(dev(np.arange(3, dtype=np.uint32), cuda))


@pytest.mark.parametrize("family", ["uniform", "normal", "normal_wide", "zipf", "multi_gaussian"])
def test_reference_query_families(bt, orc, wl, cuda, family):
    """The reference generator's query families (seeded) on u64 keys drawn
    from the same value range: both point modes against the oracle."""
    mx = 1 << 40
    g = np.random.default_rng(17)
    keys = np.unique(g.integers(0, mx, size=1 << 20, dtype=np.uint64, endpoint=True))
    vals = np.arange(len(keys), dtype=np.uint64)
    q = wl.reference_queries(family, (1 << 21) + 3, mx)
    exp = orc.point_search(keys, vals, q)
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        for mode in ("basic", "grouped"):
            assert np.array_equal(t.point_search(dev(q, cuda), mode=mode).cpu().numpy(), exp), mode
