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
        c, off, got = bt.rect_search(t, dev(x0, cuda), dev(y0, cuda), dev(x1, cuda), dev(y1, cuda))
    assert np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(off.cpu().numpy(), eo)
    assert np.array_equal(got.cpu().numpy().astype(np.uint64), ei.astype(np.uint64))


def test_rect_search_needs_32bit_keys(bt, cuda):
    import torch
    keys = np.arange(10, dtype=np.uint64)
    with bt.Tree.build(dev(keys, cuda), dev(keys, cuda)) as t:
        u = torch.zeros(1, dtype=torch.uint16, device=cuda)
        with pytest.raises(bt.BTreeError):
            bt.rect_search(t, u, u, u, u)
