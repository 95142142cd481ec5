"""ctypes wrappers of the CPU oracle and of the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, to check results.  The engine never imports it.

  Oracle   -- lib/liboracle.so (oracle.c): binary-search ground truth + literal
              restatement of the reference's page tree ("refc").
  RefHarness -- _ref/libbtref.so: the reference's own .cu sources compiled
              for sm_100a plus ref_harness.cu (needs a GPU to run).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbtref.so")
INVALID64 = np.uint64(0xFFFFFFFFFFFFFFFF)
PAGESIZE = 5000

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_I = ctypes.c_int


def build_oracle(reference=False):
    """Build lib/liboracle.so (and _ref/libbtref.so when reference=True)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if reference:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _p(a):
    return a.ctypes.data_as(_P) if a is not None else None


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_LIB):
            build_oracle()
        L = ctypes.CDLL(ORACLE_LIB)
        sig = {
            "orc_point_search": (_I, [_P, _P, _U64, _I, _I, _P, _U64, _P, _I]),
            "orc_range_count": (_I, [_P, _U64, _I, _P, _P, _U64, _P, _I]),
            "orc_range_ids": (_I, [_P, _P, _U64, _I, _I, _P, _P, _U64, _P, _P, _I]),
            "orc_bounds": (_I, [_P, _U64, _I, _P, _U64, _I, _P, _I]),
            "orc_rect_search": (_I, [_P, _P, _U64, _P, _P, _P, _P, _U64, _P, _P, _P, _I]),
            "orc_morton2_u16": (ctypes.c_uint32, [ctypes.c_uint16, ctypes.c_uint16]),
            "orc_pla_segments": (_U64, [_P, _U64, _I, ctypes.c_uint32, _U64, _I, _P, _P, _P,
                                        _U64]),
            "refc_build": (_P, [_P, _P, _U64, _P, _U64]),
            "refc_free": (None, [_P]),
            "refc_root": (_U64, [_P]),
            "refc_num_pages": (_U64, [_P]),
            "refc_point_basic": (_I, [_P, _P, _U64, _P, _I]),
            "refc_point_grouped": (_I, [_P, _P, _U64, _P, _I]),
            "refc_range_endpoint": (_I, [_P, _P, _U64, _P, _I]),
            "refc_range_count": (_I, [_P, _P, _P, _P, _P, _U64, _I, _P, _I]),
            "refc_bucket": (_I, [_U64, _I]),
            "refc_bucket2d": (_I, [_U64, _U64, _I]),
            "refc_zorder": (_U64, [_U64, _U64, _I, _I]),
            "refc_zorder_interval": (_I, [_U64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L

    # -- ground truth --------------------------------------------------------
    def point_search(self, keys, vals, queries, nthreads=0):
        keys, vals, queries = map(np.ascontiguousarray, (keys, vals, queries))
        out = np.empty(len(queries), dtype=vals.dtype)
        rc = self.L.orc_point_search(_p(keys), _p(vals), len(keys), keys.itemsize, vals.itemsize,
                                     _p(queries), len(queries), _p(out), nthreads)
        assert rc == 0
        return out

    def bounds(self, keys, queries, upper=False, nthreads=0):
        keys, queries = map(np.ascontiguousarray, (keys, queries))
        out = np.empty(len(queries), dtype=np.uint64)
        assert self.L.orc_bounds(_p(keys), len(keys), keys.itemsize, _p(queries), len(queries),
                                 int(upper), _p(out), nthreads) == 0
        return out

    def range_count(self, keys, lo, hi, nthreads=0):
        keys, lo, hi = map(np.ascontiguousarray, (keys, lo, hi))
        out = np.empty(len(lo), dtype=np.uint64)
        assert self.L.orc_range_count(_p(keys), len(keys), keys.itemsize, _p(lo), _p(hi), len(lo),
                                      _p(out), nthreads) == 0
        return out

    def range_search(self, keys, vals, lo, hi, nthreads=0):
        keys, vals, lo, hi = map(np.ascontiguousarray, (keys, vals, lo, hi))
        counts = self.range_count(keys, lo, hi, nthreads)
        offsets = np.zeros(len(lo), dtype=np.uint64)
        if len(lo) > 1:
            offsets[1:] = np.cumsum(counts[:-1], dtype=np.uint64)
        total = int(counts.sum()) if len(lo) else 0
        ids = np.empty(total, dtype=vals.dtype)
        assert self.L.orc_range_ids(_p(keys), _p(vals), len(keys), keys.itemsize, vals.itemsize,
                                    _p(lo), _p(hi), len(lo), _p(offsets), _p(ids), nthreads) == 0
        return counts, offsets, ids

    def rect_search(self, z_sorted, ids_sorted, x0, y0, x1, y1, want_ids=True, nthreads=0):
        z_sorted = np.ascontiguousarray(z_sorted, dtype=np.uint32)
        ids_sorted = np.ascontiguousarray(ids_sorted, dtype=np.uint32)
        x0, y0, x1, y1 = (np.ascontiguousarray(a, dtype=np.uint16) for a in (x0, y0, x1, y1))
        nq = len(x0)
        counts = np.empty(nq, dtype=np.uint64)
        assert self.L.orc_rect_search(_p(z_sorted), _p(ids_sorted), len(z_sorted), _p(x0), _p(y0),
                                      _p(x1), _p(y1), nq, _p(counts), None, None, nthreads) == 0
        if not want_ids:
            return counts, None, None
        offsets = np.zeros(nq, dtype=np.uint64)
        if nq > 1:
            offsets[1:] = np.cumsum(counts[:-1], dtype=np.uint64)
        ids = np.empty(int(counts.sum()), dtype=np.uint32)
        c2 = np.empty(nq, dtype=np.uint64)
        assert self.L.orc_rect_search(_p(z_sorted), _p(ids_sorted), len(z_sorted), _p(x0), _p(y0),
                                      _p(x1), _p(y1), nq, _p(c2), _p(offsets), _p(ids),
                                      nthreads) == 0
        return counts, offsets, ids

    def pla_segments(self, keys, eps, chunk=0, hull_cap=1 << 30, lines=True):
        """Error-bounded segmentation of (keys[i], i): (starts, slopes, icpts),
        or the segment count alone with lines=False (orc_pla_segments)."""
        keys = np.ascontiguousarray(keys)
        kb = keys.dtype.itemsize
        cap = min(hull_cap, len(keys) + 2)
        if not lines:
            return int(self.L.orc_pla_segments(_p(keys), len(keys), kb, eps, chunk, cap, None,
                                               None, None, 0))
        m = int(self.L.orc_pla_segments(_p(keys), len(keys), kb, eps, chunk, cap, None, None,
                                        None, 0))
        st = np.empty(m, dtype=np.uint64)
        sl = np.empty(m, dtype=np.float64)
        ic = np.empty(m, dtype=np.float64)
        self.L.orc_pla_segments(_p(keys), len(keys), kb, eps, chunk, cap, _p(st), _p(sl), _p(ic), m)
        return st, sl, ic

    def morton(self, x, y):
        return self.L.orc_morton2_u16(int(x), int(y))

    # -- literal restatement of the reference ------------------------------
    def refc_build(self, keys, data, leaf_sizes=None):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        data = np.ascontiguousarray(data, dtype=np.uint64)
        ls = None if leaf_sizes is None else np.ascontiguousarray(leaf_sizes, dtype=np.uint64)
        h = self.L.refc_build(_p(keys), _p(data), len(keys), _p(ls),
                              0 if ls is None else len(ls))
        if not h:
            raise MemoryError("refc_build failed")
        return RefcTree(self, h)

    def bucket(self, v, p):
        return self.L.refc_bucket(int(v), p)

    def bucket2d(self, a, b, p):
        return self.L.refc_bucket2d(int(a), int(b), p)

    def zorder(self, a, b, ix, iy):
        return self.L.refc_zorder(int(a), int(b), ix, iy)

    def zorder_interval(self, m):
        return self.L.refc_zorder_interval(int(m))


class RefcTree:
    def __init__(self, orc, h):
        self.o = orc
        self.h = ctypes.c_void_p(h)

    def close(self):
        if self.h:
            self.o.L.refc_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def root(self):
        return self.o.L.refc_root(self.h)

    @property
    def num_pages(self):
        return self.o.L.refc_num_pages(self.h)

    def point_basic(self, q, nthreads=0):
        q = np.ascontiguousarray(q, dtype=np.uint64)
        out = np.empty(len(q), dtype=np.uint64)
        assert self.o.L.refc_point_basic(self.h, _p(q), len(q), _p(out), nthreads) == 0
        return out

    def point_grouped(self, q, nthreads=0):
        q = np.ascontiguousarray(q, dtype=np.uint64)
        out = np.empty(len(q), dtype=np.uint64)
        assert self.o.L.refc_point_grouped(self.h, _p(q), len(q), _p(out), nthreads) == 0
        return out

    def range_endpoint(self, q, nthreads=0):
        q = np.ascontiguousarray(q, dtype=np.uint64)
        out = np.empty(len(q), dtype=np.uint64)
        assert self.o.L.refc_range_endpoint(self.h, _p(q), len(q), _p(out), nthreads) == 0
        return out

    def range_count(self, lo, hi, grouped=False, nthreads=0):
        lo = np.ascontiguousarray(lo, dtype=np.uint64)
        hi = np.ascontiguousarray(hi, dtype=np.uint64)
        elo = self.range_endpoint(lo, nthreads)
        ehi = self.range_endpoint(hi, nthreads)
        out = np.empty(len(lo), dtype=np.uint64)
        rc = self.o.L.refc_range_count(self.h, _p(lo), _p(hi), _p(elo), _p(ehi), len(lo),
                                       int(grouped), _p(out), nthreads)
        return out, rc


class RefHarness:
    """The reference implementation itself (needs a GPU and _ref/libbtref.so)."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB)
        L = ctypes.CDLL(REF_LIB)
        F = ctypes.POINTER(ctypes.c_float)
        sig = {
            "refh_build": (_I, [_P, _P, _U64]),
            "refh_free": (None, []),
            "refh_root": (_U64, []),
            "refh_point_basic": (_I, [_P, _U64, _P, F]),
            "refh_point_grouped": (_I, [_P, _U64, _P, F]),
            "refh_range_endpoints": (_I, [_P, _U64, _P]),
            "refh_range_basic": (_I, [_P, _P, _U64, _P, F]),
            "refh_range_grouped": (_I, [_I, _P, _P, _U64, _P, F]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L
        self.last_ms = 0.0

    def build(self, keys, data):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        data = np.ascontiguousarray(data, dtype=np.uint64)
        assert len(keys) % PAGESIZE == 0, "the reference needs n % 5000 == 0"
        rc = self.L.refh_build(_p(keys), _p(data), len(keys))
        assert rc == 0, f"refh_build rc={rc}"

    def free(self):
        self.L.refh_free()

    def _ms(self):
        return ctypes.c_float(0.0)

    def point_basic(self, q):
        q = np.ascontiguousarray(q, dtype=np.uint64)
        out = np.empty(len(q), dtype=np.uint64)
        ms = self._ms()
        rc = self.L.refh_point_basic(_p(q), len(q), _p(out), ctypes.byref(ms))
        assert rc == 0, f"refh_point_basic rc={rc}"
        self.last_ms = ms.value
        return out

    def point_grouped(self, q):
        """Returns (grouped queries, results in grouped order)."""
        q = np.array(q, dtype=np.uint64, copy=True)
        out = np.empty(len(q), dtype=np.uint64)
        ms = self._ms()
        rc = self.L.refh_point_grouped(_p(q), len(q), _p(out), ctypes.byref(ms))
        assert rc == 0, f"refh_point_grouped rc={rc}"
        self.last_ms = ms.value
        return q, out

    def range_endpoints(self, q):
        q = np.ascontiguousarray(q, dtype=np.uint64)
        out = np.empty(len(q), dtype=np.uint64)
        assert self.L.refh_range_endpoints(_p(q), len(q), _p(out)) == 0
        return out

    def range_basic(self, lo, hi):
        lo = np.ascontiguousarray(lo, dtype=np.uint64)
        hi = np.ascontiguousarray(hi, dtype=np.uint64)
        out = np.empty(len(lo), dtype=np.uint64)
        ms = self._ms()
        rc = self.L.refh_range_basic(_p(lo), _p(hi), len(lo), _p(out), ctypes.byref(ms))
        assert rc == 0, f"refh_range_basic rc={rc}"
        self.last_ms = ms.value
        return out

    def range_grouped(self, mode, lo, hi):
        """mode 1 = 2D grouping, 2 = Z-order.  Returns (lo, hi, counts) in grouped order."""
        lo = np.array(lo, dtype=np.uint64, copy=True)
        hi = np.array(hi, dtype=np.uint64, copy=True)
        out = np.empty(len(lo), dtype=np.uint64)
        ms = self._ms()
        rc = self.L.refh_range_grouped(mode, _p(lo), _p(hi), len(lo), _p(out), ctypes.byref(ms))
        assert rc == 0, f"refh_range_grouped rc={rc}"
        self.last_ms = ms.value
        return lo, hi, out
