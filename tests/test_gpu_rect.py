"""Rectangle search over Z-ordered points against the oracle's exact scan."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


@pytest.mark.parametrize("npts,grid,vt", [(200000, 1 << 12, np.uint32), (1 << 20, 1 << 16, np.uint32),
                                         (50000, 1 << 9, np.uint64), (1, 1 << 16, np.uint32)])
def test_rect_search_matches_oracle(bt, orc, wl, cuda, npts, grid, vt):
    g = np.random.default_rng(npts)
    x = g.integers(0, grid, size=npts).astype(np.uint16)
    y = g.integers(0, grid, size=npts).astype(np.uint16)
    z = wl.morton_u16(x, y)
    ids = np.arange(npts, dtype=vt)
    o = np.lexsort((ids, z))
    zs, idss = z[o], ids[o]
    nr = 5000
    x0 = g.integers(0, grid, size=nr).astype(np.uint16)
    y0 = g.integers(0, grid, size=nr).astype(np.uint16)
    x1 = np.minimum(x0.astype(np.int64) + g.integers(0, 257, size=nr), 65535).astype(np.uint16)
    y1 = np.minimum(y0.astype(np.int64) + g.integers(0, 257, size=nr), 65535).astype(np.uint16)
    # edge cases: whole grid, single cells, an empty box, the top corner
    x0[:4], y0[:4], x1[:4], y1[:4] = [0, 7, 9, 65000], [0, 7, 3, 65000], [65535, 7, 8, 65535], [65535, 7, 3, 65535]
    ec, eo, ei = orc.rect_search(zs, idss.astype(np.uint32), x0, y0, x1, y1)
    with bt.Tree.build(dev(zs, cuda), dev(idss, cuda)) as t:
        for mode in ("basic", "2d", "zorder"):  # box orders: outputs identical
            c, off, got = bt.rect_search(t, dev(x0, cuda), dev(y0, cuda), dev(x1, cuda),
                                         dev(y1, cuda), mode=mode)
            assert np.array_equal(c.cpu().numpy(), ec), mode
            assert np.array_equal(off.cpu().numpy(), eo), mode
            assert np.array_equal(got.cpu().numpy().astype(np.uint64), ei.astype(np.uint64)), mode


def test_rect_search_rejects_unknown_mode(bt, cuda):
    import ctypes
    import torch
    keys = np.arange(10, dtype=np.uint32)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        u = torch.zeros(1, dtype=torch.uint16, device=cuda)
        c = torch.zeros(1, dtype=torch.uint64, device=cuda)
        P = ctypes.c_void_p
        tot = ctypes.c_uint64(0)
        st = bt.lib().bt_rect_search_mode(t.handle, 7, *(P(u.data_ptr()),) * 4, 1, P(c.data_ptr()),
                                          P(c.data_ptr()), None, 0, ctypes.byref(tot), None)
        assert st == 1


def test_rect_search_needs_32bit_keys(bt, cuda):
    import torch
    keys = np.arange(10, dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        u = torch.zeros(1, dtype=torch.uint16, device=cuda)
        with pytest.raises(bt.BTreeError):
            bt.rect_search(t, u, u, u, u)


@pytest.mark.parametrize("side_log2", [0, 2, 5, 8, 11, 14, 16])
def test_rect_search_box_sizes(bt, orc, wl, cuda, side_log2):
    """Boxes whose sides reach 2^side_log2 (cell sizes from 1 to the whole
    grid), over points with duplicated coordinates."""
    g = np.random.default_rng(side_log2 + 100)
    n = 1 << 18
    x = g.integers(0, 1 << 16, size=n).astype(np.uint16)
    y = g.integers(0, 1 << 16, size=n).astype(np.uint16)
    x[: n // 8], y[: n // 8] = x[n // 8: n // 4], y[n // 8: n // 4]  # duplicate points
    z = wl.morton_u16(x, y)
    ids = np.arange(n, dtype=np.uint32)
    o = np.lexsort((ids, z))
    zs, idss = z[o], ids[o]
    nr = 3000 if side_log2 < 14 else 200
    x0 = g.integers(0, 1 << 16, size=nr)
    y0 = g.integers(0, 1 << 16, size=nr)
    x1 = np.minimum(x0 + g.integers(0, 1 << side_log2, size=nr), 65535)
    y1 = np.minimum(y0 + g.integers(0, 1 << side_log2, size=nr), 65535)
    x0, y0, x1, y1 = (a.astype(np.uint16) for a in (x0, y0, x1, y1))
    ec, eo, ei = orc.rect_search(zs, idss, x0, y0, x1, y1)
    with bt.Tree.build(dev(zs, cuda), dev(idss, cuda)) as t:
        c, off, got = bt.rect_search(t, dev(x0, cuda), dev(y0, cuda), dev(x1, cuda), dev(y1, cuda))
    assert np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(off.cpu().numpy(), eo)
    assert np.array_equal(got.cpu().numpy(), ei)


def test_rect_search_empty_tree_and_inverted_boxes(bt, cuda):
    u = lambda v: dev(np.array(v, dtype=np.uint16), cuda)  # noqa: E731
    z = np.zeros(0, dtype=np.uint32)
    with bt.Tree.build(dev(z, cuda), dev(z, cuda)) as t:
        c, off, got = bt.rect_search(t, u([0, 5]), u([0, 5]), u([65535, 9]), u([65535, 9]))
        assert c.cpu().numpy().tolist() == [0, 0] and got.numel() == 0
    z = np.arange(0, 1 << 20, 7, dtype=np.uint32)
    with bt.Tree.build(dev(z, cuda), dev(z, cuda)) as t:
        c, off, got = bt.rect_search(t, u([10, 3]), u([0, 8]), u([9, 3]), u([65535, 2]))
        assert c.cpu().numpy().tolist() == [0, 0] and got.numel() == 0
