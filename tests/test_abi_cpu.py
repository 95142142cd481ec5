"""The C-ABI library loads and exports every function include/*.h declares.

Runs without a GPU: only symbol lookup, version/status strings and argument
validation that fails before any device work.
"""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")

# The reference's public C++ API, as its own build mangles it (BPTree.h:26-55;
# checked against the reference compiled here).
REFERENCE_MANGLED = [
    "_Z12genBPlusTreePyS_ySt6vectorIySaIyEES2_RS_RyS3_S4_RP6BTPageS3_",
    "_Z29SearchingBTreeGPUOnlyOneStatePyyS_P6BTPage",
    "_Z28SearchingBTreeGPUCombineStepPyyS_P6BTPage",
    "_Z22SearchingBTreeGPURangePyS_yS_P6BTPage",
    "_Z34SearchingBTreeGPURangeWithGroupingPyS_yS_P6BTPage",
    "_Z40SearchingBTreeGPURangeWithGroupingZorderPyS_yS_P6BTPage",
]


def declared_c_functions():
    names = []
    for f in sorted(os.listdir(INCLUDE)):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(INCLUDE, f)).read()
        body = src
        if "extern \"C\" {" in src and f.endswith("_compat.h"):
            body = src[src.index("extern \"C\" {"):]
        for m in re.finditer(r"BT_API\s+[\w\s\*]+?\b(bt_\w+)\s*\(", body):
            names.append(m.group(1))
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib(bt):
    if not os.path.exists(bt.LIB_PATH):
        importlib = __import__("importlib")
        importlib.import_module("b-tree-index-searching_b200.build").build()
    return bt.lib()


def test_headers_declare_functions():
    names = declared_c_functions()
    for must in ("bt_build", "bt_point_search", "bt_range_count", "bt_range_search",
                 "bt_destroy", "bt_group_queries", "bt_compat_last_results"):
        assert must in names


def test_every_declared_symbol_exported(lib):
    missing = [n for n in declared_c_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_api_symbols_exported(bt, lib):
    h = ctypes.CDLL(bt.LIB_PATH)
    for name in REFERENCE_MANGLED:
        assert hasattr(h, name), name


def test_reference_mangling_matches_reference_build():
    """If the reference harness is built here, its own symbols agree."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libbtref.so")
    if not os.path.exists(ref):
        pytest.skip("reference harness not built")
    out = subprocess.run(["nm", "-D", "--defined-only", ref], capture_output=True, text=True).stdout
    for name in REFERENCE_MANGLED:
        assert name in out


def test_probe_library_is_separate(bt, lib):
    """The benchmark's probes live in their own library, not in the engine."""
    assert not hasattr(lib, "bt_measure_gather")
    if os.path.exists(bt.PROBE_LIB_PATH):
        p = bt.probe_lib()
        for name in ("btp_measure_gather", "btp_measure_chain", "btp_measure_hops"):
            assert hasattr(p, name)


def test_version_and_status_strings(lib):
    assert lib.bt_version() == 10000
    assert lib.bt_status_string(0) == b"ok"
    assert b"sorted" in lib.bt_status_string(2)
    assert lib.bt_status_string(99) == b"unknown status"


def test_argument_validation_without_device(lib):
    out = ctypes.c_void_p()
    # bad key width is rejected before any CUDA call
    assert lib.bt_build(None, None, 10, 3, 4, None, ctypes.byref(out)) == 1
    assert b"key_bytes" in lib.bt_last_error()
    assert lib.bt_build(None, None, 10, 4, 4, None, None) == 1
    assert lib.bt_point_search(None, 0, None, 10, None, None) == 1
    assert lib.bt_range_count(None, 0, None, None, 10, None, None) == 1
    assert lib.bt_destroy(None) == 0
    assert lib.bt_kernel_launches() == 0
