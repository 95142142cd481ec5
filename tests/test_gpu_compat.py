"""The reference's host API, run end to end.

Two programs call the compat API (include/btree_b200_compat.h, the
reference's BPTree.h:26-55 signatures) exactly as the reference's main.cu
does (main.cu:142-355):

  lib/btree                 this engine's command line (cli/btree_main.cpp):
                            the reference program's arguments and call
                            sequence; with BTREE_RESULTS_DIR set it writes the
                            outputs the reference discards, checked here
                            against the oracle;
  oracle/_ref/btree_ref_main  the reference's own main.cu and utils.cu,
                            compiled unchanged and linked against
                            libbtree_b200.so (built by `make -C oracle ref`);
                            checked through its printed self-check lines.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "b-tree-index-searching_b200", "lib", "btree")
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "btree_ref_main")


def write(path, a):
    np.ascontiguousarray(a, dtype=np.uint64).tofile(path)
    return str(path)


def run(prog, args, results_dir=None, timeout=300):
    env = dict(os.environ)
    if results_dir is not None:
        env["BTREE_RESULTS_DIR"] = str(results_dir)
    r = subprocess.run([prog] + [str(a) for a in args], capture_output=True, text=True,
                       env=env, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def load(d, name):
    return np.fromfile(os.path.join(d, name), dtype=np.uint64)


def dataset(n, seed, value_is_key):
    g = np.random.default_rng(seed)
    keys = np.unique(g.integers(1, 1 << 40, size=n + n // 8, dtype=np.uint64))[:n]
    vals = keys.copy() if value_is_key else g.integers(0, 1 << 63, size=n, dtype=np.uint64)
    order = g.permutation(n)  # the program sorts the pairs itself
    return g, keys, vals, keys[order], vals[order]


def group_order(q, max_key):
    """Stable order of the queries by their point group (the top 8 bits of
    the tree's key width), as the grouping pass forms it."""
    shift = max(0, int(max_key).bit_length() - 8)
    grp = np.minimum(q >> np.uint64(shift), np.uint64(255))
    return np.argsort(grp, kind="stable")


@pytest.fixture(scope="module")
def cli(bt):
    if not os.path.exists(CLI):
        importlib = __import__("importlib")
        importlib.import_module("b-tree-index-searching_b200.build").build()
    return CLI


@pytest.mark.parametrize("nq", [1000, (1 << 21) + 7])
@pytest.mark.parametrize("value_is_key", [True, False])
def test_cli_point_searches(cli, orc, tmp_path, nq, value_is_key):
    n = (1 << 20) + 12345
    g, keys, vals, ukeys, uvals = dataset(n, nq + value_is_key, value_is_key)
    q = g.integers(0, 1 << 41, size=nq, dtype=np.uint64)
    q[::2] = keys[g.integers(0, n, size=len(q[::2]))]
    kf, df, qf = (write(tmp_path / f, a) for f, a in (("k", ukeys), ("d", uvals), ("q", q)))
    out = run(cli, [n, kf, df, nq, qf], tmp_path)
    combined_keys = load(tmp_path, "combine_keys.bin")
    combined = load(tmp_path, "combine_results.bin")
    naive = load(tmp_path, "naive_results.bin")
    # the grouped call rewrites the caller's array into grouped order and
    # returns results in that order (BPTreeExactSearch.cu:613,722)
    assert np.array_equal(combined_keys, q[group_order(q, keys[-1])])
    assert np.array_equal(combined, orc.point_search(keys, vals, combined_keys))
    assert np.array_equal(naive, orc.point_search(keys, vals, q))
    assert "Found:" in out and "Building the Tree" in out
    if value_is_key:
        assert "Something wrong" not in out


@pytest.mark.parametrize("nr", [1000, (1 << 20) + 3])
def test_cli_range_searches(cli, orc, tmp_path, nr):
    n = 300007
    g, keys, vals, ukeys, uvals = dataset(n, nr, False)
    r = g.integers(0, n, size=nr)
    w = g.integers(1, 200, size=nr)
    lo = keys[r].copy()
    hi = keys[np.minimum(r + w - 1, n - 1)].copy()
    lo[::7] -= np.uint64(1)  # some endpoints between keys
    hi[::5] += np.uint64(1)
    files = [write(tmp_path / f, a) for f, a in (("k", ukeys), ("d", uvals), ("s", lo), ("e", hi))]
    run(cli, [n, files[0], files[1], nr, files[2], files[3]], tmp_path)
    exp = orc.range_count(keys, lo, hi)
    for mode in ("basic", "2d", "zorder"):
        assert np.array_equal(load(tmp_path, f"range_{mode}.bin"), exp), mode


def test_cli_build_only_and_bad_input(cli, tmp_path):
    g, keys, vals, ukeys, uvals = dataset(5000, 3, True)
    kf, df = write(tmp_path / "k", ukeys), write(tmp_path / "d", uvals)
    out = run(cli, [5000, kf, df])
    assert "Building the Tree" in out
    r = subprocess.run([cli, "6000", kf, df], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0  # the files hold fewer values than asked for
    r = subprocess.run([cli, "10"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "usage" in r.stderr


def test_reference_main_runs_on_the_engine(tmp_path):
    """The reference's own main.cu, unchanged, linked against the engine."""
    if not os.path.exists(REF_MAIN):
        pytest.skip("oracle/_ref/btree_ref_main not built (make -C oracle ref REF=...)")
    n, nq = 200000, 1 << 16
    g, keys, vals, ukeys, uvals = dataset(n, 11, True)  # the reference's data file is its key file
    q = keys[g.integers(0, n, size=nq)]
    kf, qf = write(tmp_path / "k", ukeys), write(tmp_path / "q", q)
    out = run(REF_MAIN, [n, kf, kf, nq, qf])
    assert out.count("Found:100% of key") == 2, out[-2000:]  # grouped and naive searches
    assert "Something wrong" not in out
    r = keys[g.integers(0, n - 100, size=nq)]
    s, e = write(tmp_path / "s", r), write(tmp_path / "e", r + np.uint64(1000))
    out = run(REF_MAIN, [n, kf, kf, nq, s, e])
    assert "Range With Grouping Zorder" in out
