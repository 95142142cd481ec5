"""Tree images: a tree written by save and read back by load searches exactly
like the original."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint64, np.uint32),
                                   (np.uint32, np.uint64), (np.uint64, np.uint64)])
@pytest.mark.parametrize("n", [0, 1, 5000, 1 << 20])
def test_save_load_round_trip(bt, orc, cuda, tmp_path, kt, vt, n):
    g = np.random.default_rng(n + 7)
    keys = np.unique(g.integers(0, int(np.iinfo(kt).max), size=n + n // 8 + 4,
                                dtype=np.uint64))[:n].astype(kt)
    vals = g.integers(0, 1 << 31, size=len(keys), dtype=np.uint64).astype(vt)
    q = g.integers(0, int(np.iinfo(kt).max), size=20000, dtype=np.uint64).astype(kt)
    if len(keys):
        q[:10000] = keys[g.integers(0, len(keys), size=10000)]
    lo = np.minimum(q, q[::-1])
    hi = np.maximum(q, q[::-1])
    path = str(tmp_path / "tree.img")
    with bt.Tree.build(dev(keys, cuda), dev(vals, cuda)) as t:
        t.save(path)
        ref_pt = t.point_search(dev(q, cuda)).cpu().numpy()
        ref_rc = t.range_count(dev(lo, cuda), dev(hi, cuda)).cpu().numpy()
    with bt.Tree.load(path) as t2:
        assert t2.info.num_keys == len(keys)
        for mode in ("basic", "grouped"):
            assert np.array_equal(t2.point_search(dev(q, cuda), mode=mode).cpu().numpy(), ref_pt)
        assert np.array_equal(t2.range_count(dev(lo, cuda), dev(hi, cuda)).cpu().numpy(), ref_rc)
    if len(keys):
        assert np.array_equal(ref_pt, orc.point_search(keys, vals, q))


def test_load_rejects_bad_files(bt, cuda, tmp_path):
    bad = tmp_path / "bad.img"
    bad.write_bytes(b"not a tree image at all" * 40)
    with pytest.raises(bt.BTreeError):
        bt.Tree.load(str(bad))
    keys = np.arange(100000, dtype=np.uint32)
    good = tmp_path / "good.img"
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        t.save(str(good))
    data = good.read_bytes()
    cut = tmp_path / "cut.img"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(bt.BTreeError):
        bt.Tree.load(str(cut))
    with pytest.raises(bt.BTreeError):
        bt.Tree.load(str(tmp_path / "missing.img"))
