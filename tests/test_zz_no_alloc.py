"""The grouped point search that allocates no device memory.

bt_point_search_grouped_noalloc exists for callers that cannot let a library
allocate device memory (their device memory is reserved by their own
allocator, or the call sits on a path where an allocation could block).  It
keeps its scratch in a fixed array inside the library.  This test calls it
through the C ABI and checks that it returns exactly what
bt_point_search(BT_POINT_GROUPED) returns, on two calls in a row (the shared
scratch keeps the previous call's contents), and that batches beyond its
limit are refused.  It lives in its own file, collected last, so that a run
stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 18


def _dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def _noalloc(bt, tree, q, out):
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return bt.lib().bt_point_search_grouped_noalloc(
        tree.handle, ctypes.c_void_p(q.data_ptr()), len(q), ctypes.c_void_p(out.data_ptr()), stream)


@pytest.mark.parametrize("kt,vt", [(np.uint32, np.uint32), (np.uint64, np.uint64)])
def test_noalloc_matches_grouped_search_twice(bt, cuda, kt, vt):
    import torch
    g = np.random.default_rng(77)
    keys = np.unique(g.integers(0, np.iinfo(kt).max, size=300000, dtype=np.uint64)).astype(kt)
    vals = g.integers(0, np.iinfo(vt).max, size=len(keys), dtype=np.uint64).astype(vt)
    with bt.Tree.build(_dev(keys, cuda), _dev(vals, cuda)) as t:
        for call, nq in enumerate((LIMIT, 100003)):  # two calls in a row, different sizes
            q = g.integers(0, np.iinfo(kt).max, size=nq, dtype=np.uint64).astype(kt)
            q[::2] = keys[g.integers(0, len(keys), size=len(q[::2]))]
            dq = _dev(q, cuda)
            expected = t.point_search(dq, mode="grouped").cpu().numpy()
            out = torch.empty(nq, dtype={4: torch.uint32, 8: torch.uint64}[t.value_bytes],
                              device=cuda)
            torch.cuda.synchronize()
            allocs = bt.lib().bt_workspace_allocations()
            assert _noalloc(bt, t, dq, out) == 0, bt.lib().bt_last_error()
            torch.cuda.synchronize()
            # the call took no scratch from the library's pool
            assert bt.lib().bt_workspace_allocations() == allocs
            assert np.array_equal(out.cpu().numpy(), expected), f"call {call}"


def test_noalloc_rejects_batches_beyond_its_limit(bt, cuda):
    import torch
    keys = np.arange(1000, dtype=np.uint32)
    with bt.Tree.build(_dev(keys, cuda), _dev(keys, cuda)) as t:
        q = torch.zeros(LIMIT + 1, dtype=torch.uint32, device=cuda)
        out = torch.empty(LIMIT + 1, dtype=torch.uint32, device=cuda)
        assert _noalloc(bt, t, q, out) == 1  # BT_ERR_INVALID_ARGUMENT
        assert b"262144" in bt.lib().bt_last_error()
