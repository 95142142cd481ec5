"""Generates tests/golden/reference_outputs.npz from the reference itself.

Runs the reference's own kernels (its .cu sources compiled for sm_100a into
oracle/_ref/libbtref.so, launched by oracle/ref_harness.cu) on small seeded
inputs and stores inputs and outputs.  Needs a GPU; the CPU test
tests/test_golden_cpu.py then checks the oracle against these vectors.

    python tests/golden/make_golden.py [out.npz]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import RefHarness  # noqa: E402

PAGESIZE = 5000


def keys_for(n, seed):
    g = np.random.default_rng(seed)
    return g, np.unique(g.integers(1, 1 << 32, size=n + n // 4, dtype=np.uint64))[:n]


def main(out):
    ref = RefHarness()
    d = {}
    # basic point search, value = rank, 2 leaves
    g, k = keys_for(2 * PAGESIZE, 1)
    v = np.arange(len(k), dtype=np.uint64)
    q = g.integers(0, 1 << 32, size=2048, dtype=np.uint64)
    q[::2] = k[g.integers(0, len(k), size=1024)]
    q[:4] = [0, k[0], k[-1], k[-1] + 1]
    ref.build(k, v)
    d.update(pb_keys=k, pb_vals=v, pb_q=q, pb_out=ref.point_basic(q))
    # grouped point search, value = key
    g, k = keys_for(2 * PAGESIZE, 2)
    q = g.integers(1, 1 << 32, size=2048, dtype=np.uint64)
    q[::2] = k[g.integers(0, len(k), size=1024)]
    ref.build(k, k)
    gq, res = ref.point_grouped(q)
    d.update(pg_keys=k, pg_q=q, pg_grouped_q=gq, pg_out=res)
    # range endpoints and counts, value = key, 3 leaves
    g, k = keys_for(3 * PAGESIZE, 3)
    r = g.integers(0, len(k), size=2048)
    w = g.integers(0, 2 * PAGESIZE, size=2048)
    lo = k[r] - g.integers(0, 2, size=2048).astype(np.uint64)
    hi = k[np.minimum(r + w, len(k) - 1)] + g.integers(0, 2, size=2048).astype(np.uint64)
    ref.build(k, k)
    d.update(rg_keys=k, rg_lo=lo, rg_hi=hi, rg_ep_lo=ref.range_endpoints(lo),
             rg_ep_hi=ref.range_endpoints(hi), rg_count=ref.range_basic(lo, hi))
    for mode, tag in ((1, "r2d"), (2, "rz")):
        glo, ghi, c = ref.range_grouped(mode, lo, hi)
        d[tag + "_lo"], d[tag + "_hi"], d[tag + "_count"] = glo, ghi, c
    ref.free()
    np.savez_compressed(out, **d)
    print("wrote", out, {kk: vv.shape for kk, vv in d.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_outputs.npz"))
