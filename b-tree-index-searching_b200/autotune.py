"""Autotuner for the search kernels' shape.

For a tree and a sample batch, times every supported (lanes per query,
rounds) configuration of the search kernels with CUDA events and keeps the
fastest.  Results do not depend on the configuration (the tests
check every one against the oracle), only speed does.  Decisions can be
cached in a JSON file keyed by (keys, key width, value width, mode, batch
size class), so a serving process tunes once per shape.

The reference has no tuning: one thread per query, 1024-thread blocks,
fanout fixed at PAGESIZE = 5000 (BPTree.h:8, BPTreeExactSearch.cu:31).  Here
the node fanout is fixed by the 128-byte line (32 u32 / 16 u64 separators);
what is tuned is how many lanes share a query below the shared-memory level
and in how many rounds a warp's 32 queries pass through those levels (that
is, how many queries each lane group keeps in flight).
"""
import json
import os
import statistics

SEARCH_CONFIGS = ((8, 1), (8, 2), (4, 1), (4, 2), (2, 1))
# learned search: (lanes per query in the index-line steps, kernel shape of
# bt_learned_set_shape: CTAs of 1024, 768, 640 or 512 threads)
LEARNED_SHAPES = ((2, 1), (2, 2), (2, 3), (2, 4))


def _key(tree, mode, nq):
    cls = max(0, int(nq).bit_length() - 1)
    return f"n{tree.info.num_keys}_k{tree.key_bytes}_v{tree.value_bytes}_{mode}_q2^{cls}"


def _time(fn, stream, repeats):
    import torch
    fn()
    fn()
    ts = []
    for _ in range(repeats):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def tune(tree, queries, mode="basic", hi=None, repeats=5, cache_path=None, configs=SEARCH_CONFIGS):
    """Pick and set the fastest search configuration for `tree` on this batch.

    mode: "basic" / "grouped" / "learned" (point search; `queries` a CUDA
    tensor), or "range" (`queries` = lo, `hi` = hi).  Returns (lanes, slots,
    {cfg: ms}); for "learned", slots is the learned kernel's shape
    (LEARNED_SHAPES).
    """
    import torch
    set_cfg = tree.set_search_config
    if mode == "learned":
        set_cfg = lambda g, i: tree.learned_set_shape(i)  # noqa: E731
    key = _key(tree, mode, len(queries))
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cached = json.load(f).get(key)
        if cached:
            set_cfg(*cached["best"])
            return cached["best"][0], cached["best"][1], cached["ms"]
    stream = torch.cuda.current_stream(queries.device)
    out = None
    if mode in ("basic", "grouped"):
        out = torch.empty(len(queries), dtype={4: torch.uint32, 8: torch.uint64}[tree.value_bytes],
                          device=queries.device)
        fn = lambda: tree.point_search(queries, mode=mode, out=out, stream=stream)  # noqa: E731
    elif mode == "learned":
        out = torch.empty(len(queries), dtype={4: torch.uint32, 8: torch.uint64}[tree.value_bytes],
                          device=queries.device)
        fn = lambda: tree.point_search(queries, mode="learned", out=out, stream=stream)  # noqa: E731
        configs = LEARNED_SHAPES
    elif mode == "range":
        out = torch.empty(len(queries), dtype=torch.uint64, device=queries.device)
        fn = lambda: tree.range_count(queries, hi, out=out, stream=stream)  # noqa: E731
    else:
        raise ValueError(mode)
    ms = {}
    for g, i in configs:
        set_cfg(g, i)
        ms[f"{g}x{i}"] = _time(fn, stream, repeats)
    best = min(ms, key=ms.get)
    g, i = (int(x) for x in best.split("x"))
    set_cfg(g, i)
    if cache_path:
        data = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                data = json.load(f)
        data[key] = {"best": [g, i], "ms": ms}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return g, i, ms


FOREST_SHAPES = ((4, 1), (8, 1), (8, 2))
FOREST_TILES = (512, 2048, 8192)
# staged-root fanouts (bt_forest_set_stage_fanout), tried at the best shape
# and tile found with the default 16
FOREST_FANOUTS = (4, 16, 64)


def _forest_key(forest, nq, nr):
    return (f"forest_t{forest.num_trees}_k{forest.key_bytes}_v{forest.value_bytes}"
            f"_q2^{max(0, int(nq).bit_length() - 1)}_r2^{max(0, int(nr).bit_length() - 1)}")


def tune_forest(forest, queries, q_offsets, out, lo=None, hi=None, r_offsets=None, counts=None,
                shapes=FOREST_SHAPES, tiles=FOREST_TILES, fanouts=FOREST_FANOUTS, repeats=3,
                flush=None, cache_path=None):
    """Pick the forest search plan's (lanes per query, rounds, tile) and the
    staged-root fanout for this batch: every (shape, tile) candidate is
    planned at fanout 16 (one captured CUDA-graph launch) and timed with CUDA
    events (an L2 flush before each timed launch when `flush`, a CUDA tensor,
    is given), then the fanouts are tried at the best of them.  Sets the
    chosen fanout on `forest` and returns (lanes, rounds, tile, fanout,
    {name: ms}); with cache_path the decision is stored and reused per forest
    and batch shape."""
    import torch
    key = _forest_key(forest, len(queries), 0 if lo is None else len(lo))
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cached = json.load(f).get(key)
        if cached:
            lanes, rounds, tile, fanout = cached["best"]
            forest.set_stage_fanout(fanout)
            return lanes, rounds, tile, fanout, cached["ms"]
    stream = torch.cuda.current_stream(queries.device)
    ms = {}

    def time_plan(lanes, rounds, tile):
        with forest.plan(queries, q_offsets, out, lo, hi, r_offsets, counts, lanes, rounds,
                         tile=tile) as p:
            p.run(stream)
            ts = []
            for _ in range(repeats):
                if flush is not None:
                    flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                p.run(stream)
                b.record(stream)
                b.synchronize()
                ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    forest.set_stage_fanout(16)
    for lanes, rounds in shapes:
        for tile in tiles:
            ms[f"{lanes}x{rounds}/t{tile}/f16"] = time_plan(lanes, rounds, tile)
    best = min(ms, key=ms.get)
    lanes, rounds = (int(x) for x in best.split("/")[0].split("x"))
    tile = int(best.split("/t")[1].split("/")[0])
    for fo in fanouts:
        name = f"{lanes}x{rounds}/t{tile}/f{fo}"
        if name not in ms:
            forest.set_stage_fanout(fo)
            ms[name] = time_plan(lanes, rounds, tile)
    best = min(ms, key=ms.get)
    fanout = int(best.split("/f")[1])
    forest.set_stage_fanout(fanout)
    if cache_path:
        data = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                data = json.load(f)
        data[key] = {"best": [lanes, rounds, tile, fanout], "ms": ms}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return lanes, rounds, tile, fanout, ms