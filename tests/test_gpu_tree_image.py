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


def test_build_from_reference_input_files(bt, orc, cuda, tmp_path):
    """Raw u64 key and data files as the reference program reads them
    (unsorted, no header); the files may hold more values than n."""
    g = np.random.default_rng(31)
    n = 200000
    keys = np.unique(g.integers(0, 1 << 63, size=n + 1000, dtype=np.uint64))[: n + 10]
    g.shuffle(keys)
    data = g.integers(0, 1 << 63, size=len(keys), dtype=np.uint64)
    kp, dp = tmp_path / "keys.bin", tmp_path / "data.bin"
    keys.tofile(kp)
    data.tofile(dp)
    q = np.concatenate([keys[g.integers(0, n, size=5000)],
                        g.integers(0, 1 << 63, size=5000, dtype=np.uint64)])
    o = np.argsort(keys[:n], kind="stable")
    exp = orc.point_search(keys[:n][o], data[:n][o], q)
    with bt.Tree.build_from_files(str(kp), str(dp), n) as t:
        assert t.info.num_keys == n
        assert np.array_equal(t.point_search(dev(q, cuda)).cpu().numpy(), exp)
    with pytest.raises(bt.BTreeError):
        bt.Tree.build_from_files(str(kp), str(dp), len(keys) + 1)
