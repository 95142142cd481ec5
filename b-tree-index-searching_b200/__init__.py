"""Python bindings (ctypes) of the B200 B+tree engine's C ABI.

The engine is the shared library ``lib/libbtree_b200.so`` (C ABI declared in
``include/btree_b200.h``).  This module only marshals pointers: device arrays
are ``torch`` CUDA tensors (plumbing for device memory and streams), host
arrays are ``numpy`` arrays.  Every search runs in the library's own kernels;
there is no Python or CPU fallback -- a missing library raises.

Mirrors the reference's host API (BPTree.h:26-55) in Python form:

    tree = Tree.build(keys, values)          # genBPlusTree
    tree.point_search(q, mode="basic")       # SearchingBTreeGPUOnlyOneState
    tree.point_search(q, mode="grouped")     # SearchingBTreeGPUCombineStep
    tree.range_count(lo, hi, mode="basic")   # SearchingBTreeGPURange
    tree.range_count(lo, hi, mode="2d")      # ...RangeWithGrouping
    tree.range_count(lo, hi, mode="zorder")  # ...RangeWithGroupingZorder
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libbtree_b200.so")

POINT_MODES = {"basic": 0, "grouped": 1, "learned": 2}
RANGE_MODES = {"basic": 0, "2d": 1, "zorder": 2}

STATUS = {
    0: "BT_OK", 1: "BT_ERR_INVALID_ARGUMENT", 2: "BT_ERR_UNSORTED",
    3: "BT_ERR_OUT_OF_MEMORY", 4: "BT_ERR_CUDA", 5: "BT_ERR_CAPACITY",
    6: "BT_ERR_NOT_SUPPORTED", 7: "BT_ERR_TIMEOUT", 8: "BT_ERR_INTERNAL",
}


class BTreeError(RuntimeError):
    """A C-ABI call returned a status other than BT_OK."""

    def __init__(self, status, where, detail):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{where}: {self.name}: {detail}")


class bt_info(ctypes.Structure):
    _fields_ = [
        ("num_keys", ctypes.c_uint64),
        ("key_bytes", ctypes.c_uint32),
        ("value_bytes", ctypes.c_uint32),
        ("num_levels", ctypes.c_uint32),
        ("fanout", ctypes.c_uint32),
        ("leaf_keys", ctypes.c_uint32),
        ("smem_levels", ctypes.c_uint32),
        ("device_bytes", ctypes.c_uint64),
        ("min_key", ctypes.c_uint64),
        ("max_key", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("values_sorted", ctypes.c_int32),
        ("lanes_per_query", ctypes.c_uint32),
        ("rounds", ctypes.c_uint32),
    ]


class bt_learned_config(ctypes.Structure):
    _fields_ = [("num_segments", ctypes.c_uint32), ("max_error", ctypes.c_uint32),
                ("hidden", ctypes.c_uint32), ("iterations", ctypes.c_uint32),
                ("learning_rate", ctypes.c_float)]


class bt_learned_report(ctypes.Structure):
    _fields_ = [("root_loss_initial", ctypes.c_float), ("root_loss_final", ctypes.c_float),
                ("root_error", ctypes.c_uint32), ("root_error_initial", ctypes.c_uint32),
                ("num_segments", ctypes.c_uint32), ("max_error", ctypes.c_uint32),
                ("eps_max", ctypes.c_uint64), ("eps_mean", ctypes.c_double),
                ("code_lines_mean", ctypes.c_double), ("index_bytes", ctypes.c_uint64),
                ("keys_per_unit", ctypes.c_uint32), ("pad", ctypes.c_uint32),
                ("train_ms", ctypes.c_double)]


class bt_server_config(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("memory_budget_bytes", ctypes.c_uint64),
                ("max_batch", ctypes.c_uint32), ("mode", ctypes.c_int32)]


class bt_server_stats(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("max_in_flight", ctypes.c_uint32),
                ("completed", ctypes.c_uint64), ("jobs", ctypes.c_uint64)]


SERVE_MODES = {"basic": 0, "grouped": 1, "learned": 2}

_lib = None

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_I = ctypes.c_int
_PROTOS = {
    "bt_version": (ctypes.c_int, []),
    "bt_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "bt_last_error": (ctypes.c_char_p, []),
    "bt_build": (_I, [_P, _P, _U64, _I, _I, _P, ctypes.POINTER(_P)]),
    "bt_build_host": (_I, [_P, _P, _U64, _I, _I, _P, ctypes.POINTER(_P)]),
    "bt_destroy": (_I, [_P]),
    "bt_get_info": (_I, [_P, ctypes.POINTER(bt_info)]),
    "bt_point_search": (_I, [_P, _I, _P, _U64, _P, _P]),
    "bt_point_search_host": (_I, [_P, _I, _P, _U64, _P, _P]),
    "bt_point_search_found": (_I, [_P, _I, _P, _U64, _P, _P, _P]),
    "bt_group_queries": (_I, [_P, _P, _U64, _P, _P, _P]),
    "bt_range_count": (_I, [_P, _I, _P, _P, _U64, _P, _P]),
    "bt_range_search": (_I, [_P, _I, _P, _P, _U64, _P, _P, _P, _U64, ctypes.POINTER(_U64), _P]),
    "bt_range_count_host": (_I, [_P, _I, _P, _P, _U64, _P, _P]),
    "bt_point_search_grouped_batch": (_I, [_P, _P, _P, _U64, _P, _P]),
    "bt_kernel_launches": (ctypes.c_uint64, []),
    "bt_workspace_allocations": (ctypes.c_uint64, []),
    "bt_partition_lookback_timeouts": (ctypes.c_uint64, []),
    "bt_sort_pairs": (_I, [_P, _P, _U64, _I, _I, _P, _P, _P]),
    "bt_build_unsorted": (_I, [_P, _P, _U64, _I, _I, _P, ctypes.POINTER(_P)]),
    "bt_save": (_I, [_P, ctypes.c_char_p]),
    "bt_build_from_files": (_I, [ctypes.c_char_p, ctypes.c_char_p, _U64, _P, ctypes.POINTER(_P)]),
    "bt_load": (_I, [ctypes.c_char_p, _P, ctypes.POINTER(_P)]),
    "bt_set_search_config": (_I, [_P, _I, _I]),
    "bt_point_search_grouped_noalloc": (_I, [_P, _P, _U64, _P, _P]),
    "bt_learned_train": (_I, [_P, ctypes.POINTER(bt_learned_config), _P,
                              ctypes.POINTER(bt_learned_report)]),
    "bt_point_search_learned": (_I, [_P, _P, _U64, _P, _P]),
    "bt_learned_last_stats": (_I, [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "bt_learned_set_shape": (_I, [_P, ctypes.c_uint32]),
    "bt_learned_last_lines": (_I, [_P, ctypes.POINTER(_U64)]),
    "bt_mlp_loss_grad": (_I, [_P, ctypes.c_uint32, _P, _P, _U64, _P, _P, _P]),
    "bt_rect_search": (_I, [_P, _P, _P, _P, _P, _U64, _P, _P, _P, _U64, ctypes.POINTER(_U64), _P]),
    "bt_rect_search_mode": (_I, [_P, _I, _P, _P, _P, _P, _U64, _P, _P, _P, _U64,
                                 ctypes.POINTER(_U64), _P]),
    "bt_forest_build": (_I, [_P, _P, _P, ctypes.c_uint32, _I, _I, _P, ctypes.POINTER(_P)]),
    "bt_forest_destroy": (_I, [_P]),
    "bt_forest_plan_create": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, ctypes.c_uint32,
                                   ctypes.POINTER(_P)]),
    "bt_forest_plan_run": (_I, [_P, _P]),
    "bt_forest_plan_destroy": (_I, [_P]),
    "bt_server_create": (_I, [_P, ctypes.POINTER(bt_server_config), ctypes.POINTER(_P)]),
    "bt_server_submit": (_I, [_P, _P, _U64, _P, ctypes.POINTER(_U64)]),
    "bt_server_wait": (_I, [_P, _U64, ctypes.POINTER(ctypes.c_double)]),
    "bt_server_get_stats": (_I, [_P, ctypes.POINTER(bt_server_stats)]),
    "bt_server_destroy": (_I, [_P]),
    "bt_server_replay": (_I, [_P, _U64, _P, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "bt_forest_set_stage_fanout": (_I, [_P, ctypes.c_uint32]),
}


def lib():
    """Load the engine library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build` "
                "(the engine has no CPU fallback)")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def _check(status, where):
    if status != 0:
        detail = lib().bt_last_error().decode(errors="replace")
        raise BTreeError(status, where, detail)


def _width(dtype):
    return np.dtype(dtype).itemsize


def _stream_ptr(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


def _is_cuda(x):
    return hasattr(x, "is_cuda") and x.is_cuda


def _torch_dtype(nbytes):
    import torch
    return {4: torch.uint32, 8: torch.uint64}[nbytes]


class Tree:
    """One B+tree in device memory, built from sorted keys."""

    def __init__(self, handle, info):
        self._h = ctypes.c_void_p(handle)
        self.info = info
        self.key_bytes = info.key_bytes
        self.value_bytes = info.value_bytes

    @classmethod
    def build(cls, keys, values, stream=None):
        """keys/values: CUDA tensors (device build) or numpy arrays (host
        build), of unsigned 4- or 8-byte integers, keys sorted ascending."""
        L = lib()
        out = ctypes.c_void_p()
        n = len(keys)
        if len(values) != n:
            raise ValueError("keys and values differ in length")
        if _is_cuda(keys):
            kb, vb = keys.element_size(), values.element_size()
            keys = keys.contiguous()
            values = values.contiguous()
            st = L.bt_build(_P(keys.data_ptr()), _P(values.data_ptr()), n, kb, vb,
                            _stream_ptr(stream), ctypes.byref(out))
        else:
            keys = np.ascontiguousarray(keys)
            values = np.ascontiguousarray(values)
            kb, vb = keys.dtype.itemsize, values.dtype.itemsize
            st = L.bt_build_host(keys.ctypes.data_as(_P), values.ctypes.data_as(_P), n, kb, vb,
                                 _stream_ptr(stream), ctypes.byref(out))
        _check(st, "bt_build")
        info = bt_info()
        _check(L.bt_get_info(out, ctypes.byref(info)), "bt_get_info")
        return cls(out.value, info)

    @classmethod
    def build_from_files(cls, keys_path, values_path, n):
        """Build from raw u64 key and value files in the reference program's
        format (bt_build_from_files)."""
        L = lib()
        out = ctypes.c_void_p()
        _check(L.bt_build_from_files(os.fsencode(keys_path), os.fsencode(values_path), n, None,
                                     ctypes.byref(out)), "bt_build_from_files")
        info = bt_info()
        _check(L.bt_get_info(out, ctypes.byref(info)), "bt_get_info")
        return cls(out.value, info)

    def save(self, path):
        """Write the built tree to one file (bt_save)."""
        _check(lib().bt_save(self._h, os.fsencode(path)), "bt_save")

    @classmethod
    def load(cls, path):
        """A tree read back from a file written by save (bt_load), on the
        current device."""
        L = lib()
        out = ctypes.c_void_p()
        _check(L.bt_load(os.fsencode(path), None, ctypes.byref(out)), "bt_load")
        info = bt_info()
        _check(L.bt_get_info(out, ctypes.byref(info)), "bt_get_info")
        return cls(out.value, info)

    @classmethod
    def build_unsorted(cls, keys, values, stream=None):
        """Build from unsorted CUDA tensors: sorted on the device first
        (bt_build_unsorted); equal keys keep their input order."""
        L = lib()
        out = ctypes.c_void_p()
        if len(values) != len(keys):
            raise ValueError("keys and values differ in length")
        keys, values = keys.contiguous(), values.contiguous()
        _check(L.bt_build_unsorted(_P(keys.data_ptr()), _P(values.data_ptr()), len(keys),
                                   keys.element_size(), values.element_size(), _stream_ptr(stream),
                                   ctypes.byref(out)), "bt_build_unsorted")
        info = bt_info()
        _check(L.bt_get_info(out, ctypes.byref(info)), "bt_get_info")
        return cls(out.value, info)

    def close(self):
        if self._h is not None and self._h.value:
            lib().bt_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_search_config(self, lanes_per_query, rounds):
        """Search kernel shape (see bt_set_search_config); results unchanged."""
        L = lib()
        _check(L.bt_set_search_config(self._h, lanes_per_query, rounds), "bt_set_search_config")
        _check(L.bt_get_info(self._h, ctypes.byref(self.info)), "bt_get_info")

    SEARCH_CONFIGS = ((8, 1), (8, 2), (4, 1), (4, 2), (2, 1))

    # -- point search ---------------------------------------------------
    def point_search_found(self, queries, mode="basic", stream=None):
        """(values, found): the values of the queried keys (all-ones on a
        miss) and a uint8 flag per query, 1 when the key is in the tree
        (bt_point_search_found).  CUDA tensors in and out, asynchronous on
        `stream`."""
        import torch
        if not _is_cuda(queries):
            raise ValueError("point_search_found takes a CUDA tensor")
        if queries.element_size() != self.key_bytes:
            raise ValueError("query width differs from the tree's key width")
        queries = queries.contiguous()
        n = len(queries)
        out = torch.empty(n, dtype=_torch_dtype(self.value_bytes), device=queries.device)
        found = torch.empty(n, dtype=torch.uint8, device=queries.device)
        _check(lib().bt_point_search_found(self._h, POINT_MODES[mode], _P(queries.data_ptr()), n,
                                           _P(out.data_ptr()), _P(found.data_ptr()),
                                           _stream_ptr(stream)), "bt_point_search_found")
        return out, found

    def point_search(self, queries, mode="basic", out=None, stream=None):
        """Values of the queried keys (all-ones on a miss), in query order.
        CUDA tensor in -> CUDA tensor out (asynchronous on `stream`);
        numpy in -> numpy out (host pipeline, synchronous)."""
        L = lib()
        m = POINT_MODES[mode]
        n = len(queries)
        if _is_cuda(queries):
            import torch
            if queries.element_size() != self.key_bytes:
                raise ValueError("query width differs from the tree's key width")
            queries = queries.contiguous()
            if out is None:
                out = torch.empty(n, dtype=_torch_dtype(self.value_bytes), device=queries.device)
            _check(L.bt_point_search(self._h, m, _P(queries.data_ptr()), n, _P(out.data_ptr()),
                                     _stream_ptr(stream)), "bt_point_search")
            return out
        queries = np.ascontiguousarray(queries)
        if queries.dtype.itemsize != self.key_bytes:
            raise ValueError("query width differs from the tree's key width")
        if out is None:
            out = np.empty(n, dtype=np.uint32 if self.value_bytes == 4 else np.uint64)
        _check(L.bt_point_search_host(self._h, m, queries.ctypes.data_as(_P), n,
                                      out.ctypes.data_as(_P), _stream_ptr(stream)),
               "bt_point_search_host")
        return out

    # -- learned position model -------------------------------------------
    def learned_train(self, num_segments=65536, max_error=0, hidden=16, iterations=400,
                      learning_rate=0.002, stream=None):
        """Build the learned index of this tree (segmentation, root training,
        unit thresholds); returns the report as a dict."""
        cfg = bt_learned_config(num_segments, max_error, hidden, iterations, learning_rate)
        rep = bt_learned_report()
        _check(lib().bt_learned_train(self._h, ctypes.byref(cfg), _stream_ptr(stream),
                                      ctypes.byref(rep)), "bt_learned_train")
        return {k: getattr(rep, k) for k, _ in bt_learned_report._fields_ if k != "pad"}

    def point_search_learned(self, queries, out=None, stream=None):
        """Point search through the learned model (same results as point_search)."""
        import torch
        n = len(queries)
        if out is None:
            out = torch.empty(n, dtype=_torch_dtype(self.value_bytes), device=queries.device)
        _check(lib().bt_point_search_learned(self._h, _P(queries.data_ptr()), n,
                                             _P(out.data_ptr()), _stream_ptr(stream)),
               "bt_point_search_learned")
        return out

    def learned_set_shape(self, shape):
        """Learned search kernel shape (bt_learned_set_shape): CTAs of 1024
        (1), 768 (2), 640 (3) or 512 (4) threads."""
        _check(lib().bt_learned_set_shape(self._h, shape), "bt_learned_set_shape")

    def learned_last_stats(self):
        """(leaf units read beyond the first, queries that took the full descent)."""
        w, f = _U64(), _U64()
        _check(lib().bt_learned_last_stats(self._h, ctypes.byref(w), ctypes.byref(f)),
               "bt_learned_last_stats")
        return w.value, f.value

    def learned_last_lines(self):
        """Code lines the last learned search counted beyond each query's first."""
        x = _U64()
        _check(lib().bt_learned_last_lines(self._h, ctypes.byref(x)), "bt_learned_last_lines")
        return x.value

    def group(self, queries, stream=None):
        """The grouping step alone: (grouped queries, caller index per slot)."""
        import torch
        n = len(queries)
        g = torch.empty_like(queries)
        perm = torch.empty(n, dtype=torch.uint32, device=queries.device)
        _check(lib().bt_group_queries(self._h, _P(queries.data_ptr()), n, _P(g.data_ptr()),
                                      _P(perm.data_ptr()), _stream_ptr(stream)), "bt_group_queries")
        return g, perm

    def search_grouped_batch(self, grouped, perm, out=None, stream=None):
        """Search a batch from group(): out[perm[i]] = value of grouped[i]."""
        import torch
        n = len(grouped)
        if out is None:
            out = torch.empty(n, dtype=_torch_dtype(self.value_bytes), device=grouped.device)
        _check(lib().bt_point_search_grouped_batch(self._h, _P(grouped.data_ptr()),
                                                   _P(perm.data_ptr()), n, _P(out.data_ptr()),
                                                   _stream_ptr(stream)),
               "bt_point_search_grouped_batch")
        return out

    # -- range search ----------------------------------------------------
    def range_count(self, lo, hi, mode="basic", out=None, stream=None):
        """Number of keys in [lo[i], hi[i]] (u64), in query order."""
        L = lib()
        m = RANGE_MODES[mode]
        n = len(lo)
        if _is_cuda(lo):
            import torch
            lo, hi = lo.contiguous(), hi.contiguous()
            if out is None:
                out = torch.empty(n, dtype=torch.uint64, device=lo.device)
            _check(L.bt_range_count(self._h, m, _P(lo.data_ptr()), _P(hi.data_ptr()), n,
                                    _P(out.data_ptr()), _stream_ptr(stream)), "bt_range_count")
            return out
        lo, hi = np.ascontiguousarray(lo), np.ascontiguousarray(hi)
        if out is None:
            out = np.empty(n, dtype=np.uint64)
        _check(L.bt_range_count_host(self._h, m, lo.ctypes.data_as(_P), hi.ctypes.data_as(_P), n,
                                     out.ctypes.data_as(_P), _stream_ptr(stream)),
               "bt_range_count_host")
        return out

    def range_search(self, lo, hi, mode="basic", ids_capacity=None, stream=None):
        """(counts, offsets, ids): ids[offsets[i]:offsets[i]+counts[i]] are the
        values of the keys in [lo[i], hi[i]], sorted ascending.  CUDA tensors."""
        import torch
        L = lib()
        m = RANGE_MODES[mode]
        n = len(lo)
        lo, hi = lo.contiguous(), hi.contiguous()
        counts = torch.empty(n, dtype=torch.uint64, device=lo.device)
        offsets = torch.empty(n, dtype=torch.uint64, device=lo.device)
        total = ctypes.c_uint64(0)
        if ids_capacity is None:
            # count first, then size the ID buffer exactly
            st = L.bt_range_search(self._h, m, _P(lo.data_ptr()), _P(hi.data_ptr()), n,
                                   _P(counts.data_ptr()), _P(offsets.data_ptr()), None, 0,
                                   ctypes.byref(total), _stream_ptr(stream))
            if st not in (0, 5):
                _check(st, "bt_range_search")
            ids_capacity = total.value
        ids = torch.empty(max(1, ids_capacity), dtype=_torch_dtype(self.value_bytes),
                          device=lo.device)
        _check(L.bt_range_search(self._h, m, _P(lo.data_ptr()), _P(hi.data_ptr()), n,
                                 _P(counts.data_ptr()), _P(offsets.data_ptr()), _P(ids.data_ptr()),
                                 ids_capacity, ctypes.byref(total), _stream_ptr(stream)),
               "bt_range_search")
        return counts, offsets, ids[: total.value]


class Forest:
    """Many independent trees built and searched together (bt_forest_*)."""

    def __init__(self, keys, values, offsets, stream=None):
        """keys/values: CUDA tensors holding every tree's sorted keys back to
        back; offsets: numpy u64 array of num_trees+1 boundaries."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.num_trees = len(off) - 1
        self.key_bytes, self.value_bytes = keys.element_size(), values.element_size()
        keys, values = keys.contiguous(), values.contiguous()
        h = ctypes.c_void_p()
        _check(lib().bt_forest_build(_P(keys.data_ptr()), _P(values.data_ptr()),
                                     off.ctypes.data_as(_P), self.num_trees, self.key_bytes,
                                     self.value_bytes, _stream_ptr(stream), ctypes.byref(h)),
               "bt_forest_build")
        self._h = h

    def set_stage_fanout(self, entries_per_descent):
        """Fanout of the shared-memory root for plans made afterwards
        (bt_forest_set_stage_fanout; default 16)."""
        _check(lib().bt_forest_set_stage_fanout(self._h, entries_per_descent),
               "bt_forest_set_stage_fanout")

    def plan(self, queries, q_offsets, out, lo=None, hi=None, r_offsets=None, counts=None,
             lanes_per_query=4, rounds=1, tile=1024):
        return ForestPlan(self, queries, q_offsets, out, lo, hi, r_offsets, counts,
                          lanes_per_query, rounds, tile)

    def close(self):
        if self._h is not None and self._h.value:
            lib().bt_forest_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ForestPlan:
    """A captured forest search (CUDA graph) over fixed buffers."""

    def __init__(self, forest, queries, q_offsets, out, lo, hi, r_offsets, counts, lanes, rounds,
                 tile):
        qo = np.ascontiguousarray(q_offsets, dtype=np.uint64)
        ro = None if r_offsets is None else np.ascontiguousarray(r_offsets, dtype=np.uint64)
        self._keep = (forest, queries, out, lo, hi, counts)
        ptr = lambda t: None if t is None else _P(t.data_ptr())  # noqa: E731
        h = ctypes.c_void_p()
        _check(lib().bt_forest_plan_create(forest._h, ptr(queries), qo.ctypes.data_as(_P), ptr(out),
                                           ptr(lo), ptr(hi),
                                           None if ro is None else ro.ctypes.data_as(_P),
                                           ptr(counts), lanes, rounds, tile, ctypes.byref(h)),
               "bt_forest_plan_create")
        self._h = h

    def run(self, stream=None):
        _check(lib().bt_forest_plan_run(self._h, _stream_ptr(stream)), "bt_forest_plan_run")

    def close(self):
        if self._h is not None and self._h.value:
            lib().bt_forest_plan_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop over one tree (see bt_server_create).
    Requests are numpy arrays; keep them (and the outputs) alive until done."""

    def __init__(self, tree, mode="basic", slots=8, memory_budget_bytes=256 << 20,
                 max_batch=65536):
        self.tree = tree
        cfg = bt_server_config(slots, memory_budget_bytes, max_batch, SERVE_MODES[mode])
        h = ctypes.c_void_p()
        _check(lib().bt_server_create(tree.handle, ctypes.byref(cfg), ctypes.byref(h)),
               "bt_server_create")
        self._h = h
        self._keep = {}

    def submit(self, queries, out=None):
        """Queue one request; returns (ticket, out array)."""
        queries = np.ascontiguousarray(queries)
        if out is None:
            out = np.empty(len(queries), dtype=np.uint32 if self.tree.value_bytes == 4 else np.uint64)
        t = _U64()
        _check(lib().bt_server_submit(self._h, queries.ctypes.data_as(_P), len(queries),
                                      out.ctypes.data_as(_P), ctypes.byref(t)), "bt_server_submit")
        self._keep[t.value] = (queries, out)
        return t.value, out

    def wait(self, ticket):
        """Block until answered; returns the latency in microseconds."""
        lat = ctypes.c_double()
        _check(lib().bt_server_wait(self._h, ticket, ctypes.byref(lat)), "bt_server_wait")
        self._keep.pop(ticket, None)
        return lat.value

    def stats(self):
        s = bt_server_stats()
        _check(lib().bt_server_get_stats(self._h, ctypes.byref(s)), "bt_server_get_stats")
        return {k: getattr(s, k) for k, _ in bt_server_stats._fields_}

    def replay(self, queries, arrival_us, outs=None):
        """Submit each request at its arrival time (us after start), wait for
        all; returns (latencies_us array, wall_us, outs)."""
        n = len(queries)
        queries = [np.ascontiguousarray(q) for q in queries]
        if outs is None:
            vt = np.uint32 if self.tree.value_bytes == 4 else np.uint64
            outs = [np.empty(len(q), dtype=vt) for q in queries]
        nq = (ctypes.c_uint64 * n)(*[len(q) for q in queries])
        qp = (ctypes.c_void_p * n)(*[q.ctypes.data for q in queries])
        op = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        lat = np.empty(n, dtype=np.float64)
        wall = ctypes.c_double()
        _check(lib().bt_server_replay(self._h, n, nq, qp, op, arr.ctypes.data_as(_P),
                                      lat.ctypes.data_as(_P), ctypes.byref(wall)),
               "bt_server_replay")
        return lat, wall.value, outs

    def close(self):
        if self._h is not None and self._h.value:
            lib().bt_server_destroy(self._h)
        self._h = None
        self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rect_search(tree, x0, y0, x1, y1, stream=None, mode="basic"):
    """Points of a Morton-keyed tree inside boxes [x0,x1] x [y0,y1] (u16 CUDA
    tensors): (counts, offsets, ids sorted per box).  mode "2d" / "zorder"
    processes the boxes grouped by the cell of their corner (same output)."""
    import torch
    L = lib()
    n = len(x0)
    m = RANGE_MODES[mode]
    x0, y0, x1, y1 = (t.contiguous() for t in (x0, y0, x1, y1))
    counts = torch.empty(n, dtype=torch.uint64, device=x0.device)
    offsets = torch.empty(n, dtype=torch.uint64, device=x0.device)
    total = ctypes.c_uint64(0)
    args = (tree.handle, m, _P(x0.data_ptr()), _P(y0.data_ptr()), _P(x1.data_ptr()),
            _P(y1.data_ptr()), n, _P(counts.data_ptr()), _P(offsets.data_ptr()))
    st = L.bt_rect_search_mode(*args, None, 0, ctypes.byref(total), _stream_ptr(stream))
    if st not in (0, 5):
        _check(st, "bt_rect_search_mode")
    ids = torch.empty(max(1, total.value), dtype=_torch_dtype(tree.value_bytes), device=x0.device)
    _check(L.bt_rect_search_mode(*args, _P(ids.data_ptr()), total.value, ctypes.byref(total),
                                 _stream_ptr(stream)), "bt_rect_search_mode")
    return counts, offsets, ids[: total.value]


def version():
    return lib().bt_version()


def kernel_launches():
    """Kernel launches issued by the library so far in this process."""
    return lib().bt_kernel_launches()


def sort_pairs(keys, values, stream=None):
    """Stable device sort of (key, value) CUDA tensors by key (bt_sort_pairs);
    returns new tensors."""
    import torch
    keys, values = keys.contiguous(), values.contiguous()
    ok, ov = torch.empty_like(keys), torch.empty_like(values)
    _check(lib().bt_sort_pairs(_P(keys.data_ptr()), _P(values.data_ptr()), len(keys),
                               keys.element_size(), values.element_size(), _P(ok.data_ptr()),
                               _P(ov.data_ptr()), _stream_ptr(stream)), "bt_sort_pairs")
    return ok, ov


PROBE_LIB_PATH = os.path.join(PKG_DIR, "lib", "libbt_probe.so")
_probe = None


def probe_lib():
    """The benchmark's memory-system probes (lib/libbt_probe.so, built from
    probe/bt_probe.cu).  A measurement aid: no search path uses it."""
    global _probe
    if _probe is None:
        if not os.path.exists(PROBE_LIB_PATH):
            raise RuntimeError(f"{PROBE_LIB_PATH} is not built (run build.py)")
        h = ctypes.CDLL(PROBE_LIB_PATH)
        h.btp_last_error.restype = ctypes.c_char_p
        h.btp_measure_gather.restype = _I
        h.btp_measure_gather.argtypes = [_U64, _U64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]
        h.btp_measure_chain.restype = _I
        h.btp_measure_chain.argtypes = [_U64, _U64, _U64, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, _I, ctypes.POINTER(ctypes.c_double)]
        h.btp_measure_hops.restype = _I
        h.btp_measure_hops.argtypes = [_U64, _U64, _U64, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_double)]
        _probe = h
    return _probe


def _probe_check(st, where):
    if st != 0:
        raise BTreeError(1, where, probe_lib().btp_last_error().decode())


def measure_gather(region_bytes, n_reads=1 << 24, block_bytes=64):
    """Random block reads per second the current GPU sustains (btp_measure_gather)."""
    r = ctypes.c_double(0)
    _probe_check(probe_lib().btp_measure_gather(region_bytes, n_reads, block_bytes, ctypes.byref(r)),
                 "btp_measure_gather")
    return r.value


def measure_chain(line_bytes, leaf_bytes, n_queries=1 << 24, leaf_read=128, lines_per_query=1,
                  in_flight=2, warm=True):
    """Queries per second of "random 128-byte line(s) from an L2-sized array,
    then one dependent random leaf read" (btp_measure_chain)."""
    r = ctypes.c_double(0)
    _probe_check(probe_lib().btp_measure_chain(line_bytes, leaf_bytes, n_queries, leaf_read,
                                               lines_per_query, in_flight, int(warm),
                                               ctypes.byref(r)), "btp_measure_chain")
    return r.value


HOP_FORMS = {"lane": 0, "pair": 1, "bulk": 2, "quad": 3, "pair_quad": 4}


def measure_hops(line_bytes, leaf_bytes, n_queries=1 << 24, hops=2, form="bulk"):
    """Queries per second of "`hops` dependent random 128-byte lines from an
    L2-sized array, then one dependent random 128-byte read from a large
    region", read by a lane per query ("lane"), a lane pair ("pair"), a lane
    whose lines arrive in shared memory by bulk copies ("bulk"), a lane quad
    ("quad"), or pairs for the lines and quads for the last read ("pair_quad")
    (btp_measure_hops)."""
    r = ctypes.c_double(0)
    _probe_check(probe_lib().btp_measure_hops(line_bytes, leaf_bytes, n_queries, hops,
                                              HOP_FORMS[form], ctypes.byref(r)), "btp_measure_hops")
    return r.value
