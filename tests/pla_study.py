"""Segments an error-bounded linear segmentation needs on the learned-index
keys (2^28 u64 keys, the cumulative sum of floor(lognormal(4, 2)) + 1 gaps).

    python tests/pla_study.py [keys_log2]      # default 28; about 2 minutes

Prints, for each bound eps, the number of segments of the optimal greedy
segmentation (oracle.orc_pla_segments: O'Rourke's streaming fit, the
PGM-index's segmentation) without chunking and with the engine's chunking
(segments never cross a multiple of 2^14 keys), and the least eps whose
chunked segmentation fits in 2^16 segments.  Not collected by pytest (the
oracle tests pin the segmentation itself on small inputs).
"""
import importlib
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle.oracle import Oracle  # noqa: E402

CHUNK = 1 << 14


def main(keys_log2=28):
    wl = importlib.import_module("b-tree-index-searching_b200.workloads")
    keys = wl.lognormal_keys(1 << keys_log2)
    orc = Oracle()
    print(f"{len(keys)} keys")
    print("eps  segments(optimal)  segments(chunked 2^14)  keys/segment")
    for eps in (16, 32, 64, 128, 181, 256, 512):
        a = orc.pla_segments(keys, eps, lines=False)
        b = orc.pla_segments(keys, eps, chunk=CHUNK, hull_cap=32, lines=False)
        print(f"{eps:4d} {a:18d} {b:23d} {len(keys) / b:13.1f}")
    lo, hi = 1, 1 << 16
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if orc.pla_segments(keys, mid, chunk=CHUNK, hull_cap=32, lines=False) <= 1 << 16:
            hi = mid
        else:
            lo = mid
    print(f"least eps with at most 2^16 segments (chunked): {hi}")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 28)
