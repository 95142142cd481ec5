#!/usr/bin/env python
"""Benchmark of the B200 B+tree engine.

Default workload (one "step" = one batched point search through the learned
index): 2^28 unique u64 keys, the cumulative sum of floor(lognormal(4, 2)) + 1
gaps (value = rank), bulk-built once with a learned index of 2^16 leaf
segments trained on the GPU; a batch of 2^24 point queries, 90% keys drawn
uniformly over the ranks, 10% uniform in [min, max].

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line on rank 0.  `value` is whole-job queries/s of the learned
search with the queries resident in HBM (device-timed with CUDA events, max
over ranks); `plain` is the same batch through the plain tree search, and
`learned_over_plain` their ratio; `plain_grouped` the reference's batched
path (radix grouping + grouped search, the grouping timed) on the same batch
and `learned_over_plain_grouped` that ratio; `e2e` is the learned search through the
host-buffer C-ABI call bt_point_search_host(BT_POINT_LEARNED) (H2D of the
queries and D2H of the results inside the timed region).  The path shards as
independent replicas (every rank holds the tree and answers its own batch, no
collective on the data path), so N GPUs report weak scaling.  `--impl
reference` times the CPU restatement of the reference's algorithm (its
fanout-5000 page tree, oracle/oracle.c) on the host cores, on the same
workload.  Further objects: the reference's own kernels on this GPU
(`reference_gpu`), the radix-grouped configuration (`grouped`), the
L2-resident basic search (`small`), ranges, rectangles, the forest, the
build and the request loop (`serving`).
"""
import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "b-tree-index-searching_b200"
METRIC = "point & range queries/sec on 1 B200, plain vs batched+learned; p99 latency"
L2_FLUSH_BYTES = 512 << 20


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--keys-log2", type=int, default=28, help="keys of the learned-index workload")
    p.add_argument("--queries-log2", type=int, default=24)
    p.add_argument("--grouped-keys-log2", type=int, default=26,
                   help="keys of the radix-grouped workload (u32)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-log2", type=int, default=22)
    p.add_argument("--segments-log2", type=int, default=16, help="learned index segments")
    p.add_argument("--no-serving", action="store_true", help="skip the request loop")
    p.add_argument("--no-grouped", action="store_true", help="skip the radix-grouped section")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip timing the reference's own kernels")
    p.add_argument("--serve-requests", type=int, default=3000)
    p.add_argument("--serve-rate", type=float, default=20000.0, help="requests per second")
    p.add_argument("--no-forest", action="store_true", help="skip the 4096-tree forest section")
    p.add_argument("--no-rect", action="store_true", help="skip the rectangle-search section")
    p.add_argument("--rect-boxes-log2", type=int, default=20, help="boxes in the rectangle section")
    p.add_argument("--forest-trees", type=int, default=4096, help="trees in the forest section")
    p.add_argument("--only", choices=["learned", "learned_kernel", "grouped", "ranges", "forest",
                                      "rect", "small"],
                   help="run one extension section alone on cuda:0 and print its JSON object "
                        "(for profiling; not the bench line)")
    return p.parse_args(argv)


# ----------------------------------------------------------------- ranks ----

def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_dist(world, local_rank, backend="nccl"):
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return dist


def max_over_ranks(x, dist, device=None):
    """Max of a float over all ranks (the job's time is its slowest rank)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ---------------------------------------------------------------- clocks ----

class ClockSampler:
    """nvidia-smi samples (100 ms) of the local GPU around the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons, n = [], None, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                n += 1
                for name, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": n}


# -------------------------------------------------------------- workload ----

def _cached(tag, make):
    cache = os.path.join(tempfile.gettempdir(), "btree_b200_bench")
    os.makedirs(cache, exist_ok=True)
    f = os.path.join(cache, tag + ".npz")
    if os.path.exists(f):
        d = np.load(f)
        return d["keys"], d["vals"], d["q"]
    keys, vals, q = make()
    np.savez(f, keys=keys, vals=vals, q=q)
    return keys, vals, q


def lognormal_workload(keys_log2, queries_log2, rank):
    """The learned-index workload; each replica answers its own batch."""
    wl = importlib.import_module(PKG + ".workloads")
    qs = None if rank == 0 else wl.KEY_SEED + 7 + 100 * rank
    return _cached(f"lognormal_k{keys_log2}_q{queries_log2}_r{rank}",
                   lambda: wl.lognormal_point(1 << keys_log2, 1 << queries_log2, query_seed=qs))


def zipf_workload(keys_log2, queries_log2, rank):
    """The radix-grouped workload; each replica answers its own batch."""
    wl = importlib.import_module(PKG + ".workloads")

    def make():
        keys, vals, q = wl.point_zipf(1 << keys_log2, 1 << queries_log2, seed=wl.KEY_SEED)
        if rank:
            _, _, q = wl.point_zipf(1 << keys_log2, 1 << queries_log2, seed=wl.KEY_SEED + 100 * rank)
        return keys, vals, q
    return _cached(f"zipf_k{keys_log2}_q{queries_log2}_r{rank}", make)


def workload_desc(args):
    return {
        "workload": (f"batched+learned point search: 2^{args.keys_log2} unique u64 keys = "
                     "cumsum(floor(lognormal(4, 2)) + 1) (value = rank), learned index of "
                     f"2^{args.segments_log2} segments; batches of 2^{args.queries_log2} queries, "
                     "90% keys uniform over the ranks, 10% uniform in [min, max]"),
        "keys": 1 << args.keys_log2,
        "queries_per_step": 1 << args.queries_log2,
        "key_type": "u64", "value_type": "u64",
        "l2": "flushed before every timed step (512 MiB write); tree (4.5 GiB) > L2",
        "parallelism": f"replicas x{args.gpus}",
    }


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)[name]
        return float(d["bytes_per_query"])
    except (OSError, KeyError, ValueError):
        return None


# ------------------------------------------------------------ cpu leg -------

def cpu_refc_qps(keys, vals, q, sample_log2, gpu_res=None, repeats=3):
    """The reference's algorithm on the host cores: its fanout-5000 page tree
    restated in C (oracle/oracle.c refc_*), OpenMP over all cores.  The
    binary-search oracle's answers for the same sample (the secondary timing)
    are also compared with the GPU results `gpu_res`."""
    from oracle.oracle import Oracle
    orc = Oracle()
    t = orc.refc_build(keys.astype(np.uint64), vals.astype(np.uint64))
    qs = q[: min(len(q), 1 << sample_log2)].astype(np.uint64)
    best = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        t.point_basic(qs)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    t.close()
    # lower_bound over the sorted array, same sample (secondary figure)
    t0 = time.perf_counter()
    exp = orc.point_search(keys, vals, q[: len(qs)])
    lb = len(qs) / (time.perf_counter() - t0)
    matches = None if gpu_res is None else bool(np.array_equal(gpu_res[: len(qs)], exp))
    return len(qs) / best, lb, len(qs), matches


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    keys, vals, q = lognormal_workload(args.keys_log2, args.queries_log2, 0)
    from oracle.oracle import Oracle
    orc = Oracle()
    t = orc.refc_build(keys.astype(np.uint64), vals.astype(np.uint64))
    sample = min(len(q), 1 << args.cpu_sample_log2)
    qs = q[:sample].astype(np.uint64)
    for _ in range(args.warmup):
        t.point_basic(qs)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        t.point_basic(qs)
        times.append(time.perf_counter() - t0)
    t.close()
    ms = 1000.0 * statistics.mean(times)
    qps = sample / statistics.mean(times)
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded)", "config": workload_desc(args),
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} of the step's queries per step, reference page "
                                   "tree (fanout 5000) restated in C, OpenMP on all cores"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------- request loop ----

def serving_section(args, bt, tree, keys, plain_cfg, learned_cfg):
    """Poisson request loop on the learned-index tree: batch sizes round(2^U),
    U ~ uniform[0, 16], 90% hits uniform over the ranks, 10% uniform in
    [min, max]; pinned host buffers; p50/p99 from arrival to completion,
    plain and learned."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    g = wl.rng(wl.KEY_SEED + 9)
    n = len(keys)
    sizes = np.rint(2.0 ** g.uniform(0, 16, size=args.serve_requests)).astype(np.int64)
    reqs = []
    for m in sizes:
        r = keys[g.integers(0, n, size=m)]
        mm = g.random(m) < 0.10
        r[mm] = g.integers(int(keys[0]), int(keys[-1]) + 1, size=int(mm.sum()), dtype=np.uint64)
        reqs.append(torch.from_numpy(r).pin_memory().numpy())
    outs = [torch.empty(len(r), dtype=torch.uint64).pin_memory().numpy() for r in reqs]
    arrivals = np.cumsum(g.exponential(1e6 / args.serve_rate, size=len(reqs)))
    res = {"requests": int(len(reqs)), "rate_per_s": args.serve_rate,
           "batch_sizes": "round(2^U), U ~ uniform[0,16]"}
    for mode in ("basic", "learned"):
        tree.set_search_config(*(learned_cfg if mode == "learned" else plain_cfg))
        with bt.Server(tree, mode=mode, slots=8, memory_budget_bytes=512 << 20) as srv:
            srv.replay(reqs, arrivals - arrivals[0], outs)  # warm-up: the whole loop once
            lat, wall, _ = srv.replay(reqs, arrivals - arrivals[0], outs)
            st = srv.stats()
        res["plain" if mode == "basic" else "learned"] = {
            "p50_us": float(np.percentile(lat, 50)), "p99_us": float(np.percentile(lat, 99)),
            "max_us": float(lat.max()), "over_1ms": int(np.count_nonzero(lat > 1000.0)),
            "mean_us": float(lat.mean()), "queries_per_s": float(sizes.sum() / (wall / 1e6)),
            "max_in_flight": st["max_in_flight"], "slots": st["slots"]}
    return res


# ------------------------------------------------ forest and rectangles ----

def _timed_ms(fn, stream, flush, steps):
    import torch
    ts = []
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.mean(ts)


def forest_section(args, device, bt, flush):
    """Batched uneven forest workload: 4096 trees of round(2^U), U ~ [10, 20], u32
    keys; per tree round(2^U), U ~ [6, 16], point queries (80% hits) plus 1%
    range queries of width [1, 2^12] ranks; every batch is one launch of a
    captured CUDA graph.  The plan's lanes/rounds and tile come from the
    autotuner (autotune.tune_forest)."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    keys, vals, koff, q, qoff, lo, hi, roff = wl.forest(num_trees=args.forest_trees)
    stream = torch.cuda.current_stream(device)
    f = bt.Forest(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device), koff)
    dq = torch.from_numpy(q).to(device)
    dlo, dhi = torch.from_numpy(lo).to(device), torch.from_numpy(hi).to(device)
    out = torch.empty(len(q), dtype=torch.uint32, device=device)
    counts = torch.empty(len(lo), dtype=torch.uint64, device=device)
    at = importlib.import_module(PKG + ".autotune")
    lanes, rounds, tile, fanout, tried = at.tune_forest(f, dq, qoff, out, dlo, dhi, roff, counts,
                                                        flush=flush)
    with f.plan(dq, qoff, out, dlo, dhi, roff, counts, lanes, rounds, tile=tile) as p:
        l0 = bt.kernel_launches()
        ms = _timed_ms(lambda: p.run(stream), stream, flush, args.steps)
        launches = (bt.kernel_launches() - l0) / args.steps
    res, cnt = out.cpu().numpy(), counts.cpu().numpy()
    f.close()
    # properties of the answers (exactness itself is the forest tests' job):
    # a found value is the key's rank, so it must point back at the query; a
    # query that was drawn from the keys must be found; a range [key[a],
    # key[b]] over unique keys holds b - a + 1 keys
    sizes = np.diff(koff.astype(np.int64))
    tq = np.repeat(np.arange(len(sizes)), np.diff(qoff.astype(np.int64)))
    found = res != np.uint32(0xFFFFFFFF)
    ok = bool(np.all(res[found] < sizes[tq[found]]))
    ok = ok and bool(np.array_equal(keys[koff[tq[found]].astype(np.int64) + res[found]], q[found]))
    pos = np.searchsorted
    miss = ~found
    ok = ok and not any(np.isin(q[miss][tq[miss] == t], keys[koff[t]:koff[t + 1]]).any()
                        for t in range(0, len(sizes), 257))
    tr = np.repeat(np.arange(len(sizes)), np.diff(roff.astype(np.int64)))
    exp_cnt = np.empty(len(lo), dtype=np.int64)
    for t in range(len(sizes)):
        k = keys[koff[t]:koff[t + 1]]
        s = slice(int(roff[t]), int(roff[t + 1]))
        exp_cnt[s] = pos(k, hi[s], side="right") - pos(k, lo[s], side="left")
    ok = ok and bool(np.array_equal(cnt.astype(np.int64), exp_cnt))
    total = len(q) + len(lo)
    hits = int(np.count_nonzero(res != np.uint32(0xFFFFFFFF)))
    alg = len(q) * (4 + 4 + 32) + hits * 32 + len(lo) * (2 * 4 + 8 + 2 * 32)
    peak, _ = measured_peak()
    return {
        "workload": (f"{len(koff) - 1} trees, {len(keys)} u32 keys in total (sizes round(2^U), "
                     f"U~[10,20]); {len(q)} point queries (80% hits) + {len(lo)} range queries"),
        "value": total / (ms / 1e3), "unit": "queries/s", "ms_per_batch": ms,
        "graph_launches_per_batch": launches, "lanes_per_query": lanes, "rounds": rounds,
        "tile": tile, "stage_fanout": fanout, "autotune_ms": tried, "answers_consistent": ok,
        "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak},
    }


def build_section(device, bt, keys, vals):
    """Bulk build of the benchmark tree from device-resident pairs: from
    sorted keys (bt_build), and from the same pairs shuffled (bt_build_unsorted:
    device radix sort, then the build).  Wall time around the synchronous
    calls, best of three."""
    import torch
    dk = torch.from_numpy(keys).to(device)
    dv = torch.from_numpy(vals).to(device)
    perm = np.random.default_rng(5).permutation(len(keys))
    uk = torch.from_numpy(keys[perm]).to(device)
    uv = torch.from_numpy(vals[perm]).to(device)

    def best(fn):
        ts = []
        for _ in range(3):
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            t = fn()
            torch.cuda.synchronize(device)
            ts.append(time.perf_counter() - t0)
            t.close()
        return 1e3 * min(ts)

    sorted_ms = best(lambda: bt.Tree.build(dk, dv))
    unsorted_ms = best(lambda: bt.Tree.build_unsorted(uk, uv))
    # the device sort alone, event-timed (its scratch comes from the engine's
    # cached pool after the first call; no allocation in the timed region)
    stream = torch.cuda.current_stream(device)
    ok_, ov_ = torch.empty_like(uk), torch.empty_like(uv)
    P = ctypes.c_void_p
    sort = lambda: bt._check(bt.lib().bt_sort_pairs(  # noqa: E731
        P(uk.data_ptr()), P(uv.data_ptr()), len(keys), uk.element_size(), uv.element_size(),
        P(ok_.data_ptr()), P(ov_.data_ptr()), P(stream.cuda_stream)), "sort")
    sort()
    sort_ms = _timed_ms(sort, stream, torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device), 5)
    return {"keys": len(keys), "sorted_ms": sorted_ms, "unsorted_ms": unsorted_ms,
            "timing": "wall clock around the synchronous calls, the cudaMalloc of the tree "
                      "included; sort_ms: CUDA events around bt_sort_pairs alone",
            "sort_ms": sort_ms, "pairs_per_s_sort": len(keys) / (sort_ms / 1e3),
            "keys_per_s_sorted": len(keys) / (sorted_ms / 1e3),
            "keys_per_s_unsorted": len(keys) / (unsorted_ms / 1e3)}


def range_section(args, device, bt, flush, tree, keys):
    """Range search on the benchmark tree (2^26 u32 keys, value = rank): 2^22
    ranges [key[r], key[min(r + w - 1, n - 1)]], r uniform, w uniform in
    [1, 64] ranks.  Counts in the three modes of the reference (basic, 2-D
    grouped, Z-order grouped; grouping included in the time), and counts plus
    hit IDs (values ascend with keys here, so no sort)."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    nr = 1 << 22
    lo, hi = wl.range_queries(keys, nr, 64)
    stream = torch.cuda.current_stream(device)
    dlo, dhi = torch.from_numpy(lo).to(device), torch.from_numpy(hi).to(device)
    cnt = torch.empty(nr, dtype=torch.uint64, device=device)
    at = importlib.import_module(PKG + ".autotune")
    r_lanes, r_rounds, r_ms = at.tune(tree, dlo, mode="range", hi=dhi, repeats=3)
    res = {}
    counts_ref = None
    for mode in ("basic", "2d", "zorder"):
        tree.range_count(dlo, dhi, mode=mode, out=cnt, stream=stream)
        ms = _timed_ms(lambda: tree.range_count(dlo, dhi, mode=mode, out=cnt, stream=stream),
                       stream, flush, max(3, args.steps))
        c = cnt.cpu().numpy()
        if counts_ref is None:
            counts_ref = c
        res[mode] = {"ranges_per_s": nr / (ms / 1e3), "ms": ms,
                     "same_counts_as_basic": bool(np.array_equal(c, counts_ref))}
    # with unique keys and value = rank, the count of [key[r], key[e]] is e - r + 1
    r_idx = np.searchsorted(keys, lo)
    e_idx = np.searchsorted(keys, hi)
    counts_ok = bool(np.array_equal(counts_ref.astype(np.int64), e_idx - r_idx + 1))
    hits = int(counts_ref.sum())
    tree.range_search(dlo, dhi, mode="basic", ids_capacity=hits)
    ms_ids = _timed_ms(lambda: tree.range_search(dlo, dhi, mode="basic", ids_capacity=hits,
                                                 stream=stream),
                       stream, flush, max(3, args.steps // 3))
    peak, _ = measured_peak()
    alg = nr * (2 * 4 + 8 + 2 * 32)  # both bounds' keys in, count out, two key sectors
    base_ms = res["basic"]["ms"]
    return {
        "workload": "2^26 u32 keys (value = rank), 2^22 ranges of width uniform [1, 64] ranks",
        "counts": res, "counts_equal_rank_difference": counts_ok,
        "autotune": {"lanes_per_query": r_lanes, "rounds": r_rounds, "ms": r_ms},
        "ids": {"ranges_per_s": nr / (ms_ids / 1e3), "ms": ms_ids, "hits": hits,
                "api": "Tree.range_search (counts, scan, offsets, ID fill)"},
        "roofline": {"bound": "hbm", "kernel": "bounds_line_kernel (basic counts)",
                     "achieved": alg / (base_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (base_ms / 1e3) / 1e9 / peak},
    }


def rect_section(args, device, bt, flush):
    """Rectangle workload: 2^24 points (x, y uniform u16) keyed by their
    32-bit Morton code (value = point ID, sorted by (code, ID)); 2^20
    rectangles with a uniform corner and sides uniform in [1, 256].  Timed:
    one bt_rect_search_mode call (box grouping, count pass, scan, fill pass,
    per-box ID sort) into a buffer sized by an untimed first call, with the
    boxes in 2-D-grouped, Z-order-grouped and input order; beside it the reference's
    own formulation, hit counts of the Z interval [Z(x0,y0), Z(x1,y1)] under
    the 2-D-grouped and Z-order-grouped range modes."""
    import ctypes
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    z, ids, x0, y0, x1, y1 = wl.zorder_points(n_rects=1 << args.rect_boxes_log2)
    stream = torch.cuda.current_stream(device)
    tree = bt.Tree.build(torch.from_numpy(z).to(device), torch.from_numpy(ids).to(device))
    d = [torch.from_numpy(a).to(device) for a in (x0, y0, x1, y1)]
    counts, offsets, hits = bt.rect_search(tree, *d)  # sizes the ID buffer
    total = ctypes.c_uint64(0)
    P = ctypes.c_void_p
    rsteps = max(3, args.steps // 3)
    by_mode = {}
    for mname, m in (("2d", 1), ("zorder", 2), ("basic", 0)):
        cargs = (tree.handle, m, *(P(t.data_ptr()) for t in d), len(x0), P(counts.data_ptr()),
                 P(offsets.data_ptr()), P(hits.data_ptr()), len(hits), ctypes.byref(total),
                 P(stream.cuda_stream))

        def run():
            st = bt.lib().bt_rect_search_mode(*cargs)
            if st != 0:
                raise RuntimeError(f"bt_rect_search_mode failed with status {st}")

        run()
        l0 = bt.kernel_launches()
        mms = _timed_ms(run, stream, flush, rsteps)
        by_mode[mname] = {"rects_per_s": len(x0) / (mms / 1e3), "ms": mms,
                          "launches_per_call": (bt.kernel_launches() - l0) / rsteps}
        if mname == "2d":
            ref_c, ref_got = counts.cpu().numpy(), hits.cpu().numpy()
        else:
            by_mode[mname]["same_output_as_2d"] = bool(
                np.array_equal(counts.cpu().numpy(), ref_c) and np.array_equal(hits.cpu().numpy(), ref_got))
    best = min(by_mode, key=lambda k: by_mode[k]["ms"])
    ms = by_mode[best]["ms"]
    launches = by_mode[best]["launches_per_call"]
    c, off, got = counts.cpu().numpy(), offsets.cpu().numpy(), hits.cpu().numpy()
    # properties of the first 2048 answers (exactness is the rectangle tests'
    # job): IDs strictly ascending per box and every hit inside its box
    zid = np.empty(len(z), dtype=np.uint32)
    zid[ids] = z
    ok = True
    for i in range(min(2048, len(x0))):
        h = got[int(off[i]):int(off[i] + c[i])]
        hz = zid[h]
        hx, hy = (wl.compact_u16(hz), wl.compact_u16(hz >> np.uint32(1)))
        ok = ok and bool(np.all(np.diff(h.astype(np.int64)) > 0)) and bool(
            np.all((hx >= x0[i]) & (hx <= x1[i]) & (hy >= y0[i]) & (hy <= y1[i])))
    zl = torch.from_numpy(wl.morton_u16(x0, y0)).to(device)
    zh = torch.from_numpy(wl.morton_u16(x1, y1)).to(device)
    cnt = torch.empty(len(x0), dtype=torch.uint64, device=device)
    zi = {}
    for mode in ("2d", "zorder"):
        zms = _timed_ms(lambda: tree.range_count(zl, zh, mode=mode, out=cnt, stream=stream),
                        stream, flush, 3)
        zi[mode] = {"rects_per_s": len(x0) / (zms / 1e3), "ms": zms,
                    "interval_hits": int(cnt.sum().item())}
    tree.close()
    nh = int(c.sum())
    # per box: its corners (8 B), count and offset out (16 B), one 32-byte
    # key sector for the descent; per hit: key read, ID read, ID write
    alg = len(x0) * (8 + 16 + 32) + nh * (4 + 4 + 4)
    peak, _ = measured_peak()
    return {
        "workload": "2^24 points (u16 x, y; 32-bit Morton keys, value = ID), 2^20 rectangles, "
                    "sides uniform [1, 256]; counts + sorted hit IDs",
        "value": len(x0) / (ms / 1e3), "unit": "rectangles/s", "ms": ms, "launches_per_call": launches,
        "mode": best, "modes": by_mode,
        "hits": nh, "hits_per_rect": nh / len(x0), "answers_consistent_first_2048": ok,
        "z_interval_counts": zi,
        "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak},
    }


# ------------------------------------------- radix-grouped configuration ----

def grouped_section(args, device, bt, flush, stream, rank=0):
    """Radix-grouped point search (2^26 unique uniform u32 keys, value =
    rank; 2^24 queries, 90% keys by Zipf(0.99) rank through a random rank
    permutation, 10% uniform u32; grouped by the top 8 key bits, then
    searched), beside the ungrouped basic search of the same batch and the
    grouped search through the host-buffer C-ABI call.  Returns the section
    and the tree (for the range section) and its keys."""
    import torch
    L = bt.lib()
    keys, vals, q = zipf_workload(args.grouped_keys_log2, args.queries_log2, rank)
    nq = len(q)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    dq = torch.from_numpy(q).to(device)
    grouped = torch.empty_like(dq)
    perm = torch.empty(nq, dtype=torch.uint32, device=device)
    out = torch.empty(nq, dtype=torch.uint32, device=device)
    P = ctypes.c_void_p
    sp = P(stream.cuda_stream)
    at = importlib.import_module(PKG + ".autotune")
    b_lanes, b_slots, _ = at.tune(tree, dq, mode="basic", repeats=3)
    g_lanes, g_slots, _ = at.tune(tree, dq, mode="grouped", repeats=3)
    tree.set_search_config(g_lanes, g_slots)

    def group_into():
        bt._check(L.bt_group_queries(tree.handle, P(dq.data_ptr()), nq, P(grouped.data_ptr()),
                                     P(perm.data_ptr()), sp), "group")

    def search_grouped():
        bt._check(L.bt_point_search_grouped_batch(tree.handle, P(grouped.data_ptr()),
                                                  P(perm.data_ptr()), nq, P(out.data_ptr()), sp),
                  "search")

    for _ in range(3):
        group_into()
        search_grouped()
    torch.cuda.synchronize(device)
    res = out.cpu().numpy()
    hits = int(np.count_nonzero(res != np.uint32(0xFFFFFFFF)))
    steps = max(3, args.steps)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        group_into()
        ev[i][1].record(stream)
        search_grouped()
        ev[i][2].record(stream)
    torch.cuda.synchronize(device)
    step_ms = statistics.mean(e[0].elapsed_time(e[2]) for e in ev)
    search_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    group_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    tree.set_search_config(b_lanes, b_slots)
    basic_ms = _timed_ms(lambda: bt._check(L.bt_point_search(tree.handle, 0, P(dq.data_ptr()), nq,
                                                             P(out.data_ptr()), sp), "basic"),
                         stream, flush, steps)
    # end to end: the grouped search through host buffers
    tree.set_search_config(g_lanes, g_slots)
    hq = torch.from_numpy(q).pin_memory()
    hout = torch.empty(nq, dtype=torch.uint32).pin_memory()
    hq_p, hout_p = P(hq.data_ptr()), P(hout.data_ptr())
    for _ in range(2):
        bt._check(L.bt_point_search_host(tree.handle, 1, hq_p, nq, hout_p, sp), "e2e")
    e2e_t = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        bt._check(L.bt_point_search_host(tree.handle, 1, hq_p, nq, hout_p, sp), "e2e")
        e2e_t.append(time.perf_counter() - t0)
    kb = vb = 4
    alg = nq * (kb + vb + 32) + hits * 32
    peak, _ = measured_peak()
    leaf_bytes = -(-len(keys) // (32 // kb)) * 64
    gather_rps = bt.measure_gather(leaf_bytes, 1 << 24, 64)
    tq = profiled_traffic("point_kernel_grouped_zipf_k26_q24")
    sec = {
        "workload": (f"radix-grouped point search: 2^{args.grouped_keys_log2} unique uniform u32 "
                     f"keys (value = rank), batches of 2^{args.queries_log2} queries, 90% keys by "
                     "Zipf(0.99) rank, 10% uniform u32; grouped by the top 8 key bits"),
        "value": nq / (step_ms / 1e3), "unit": "queries/s", "ms_per_step": step_ms,
        "breakdown_ms": {"group": group_ms, "search": search_ms},
        "plain_basic": {"value": nq / (basic_ms / 1e3), "unit": "queries/s", "ms": basic_ms},
        "e2e": {"value": nq / statistics.mean(e2e_t), "unit": "queries/s",
                "h2d_bytes_per_step": nq * kb, "d2h_bytes_per_step": nq * vb,
                "api": "bt_point_search_host (grouped), pinned host buffers",
                "matches_device_result": bool(np.array_equal(hout.numpy(), res))},
        "roofline": {"bound": "hbm", "kernel": "point_window_kernel (grouped batch)",
                     "achieved": alg / (search_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (search_ms / 1e3) / 1e9 / peak,
                     "traffic": None if tq is None else tq * nq,
                     "traffic_source": "not measured in this run: ncu DRAM bytes per query of "
                                       "the grouped search kernel from a 2^22-query capture "
                                       "(profiles/search_kernels_zipf_k26_q22.md) x queries",
                     "random_gather_ceiling": {"reads_per_s": gather_rps, "block_bytes": 64,
                                               "frac": nq / (search_ms / 1e3) / gather_rps}},
        "autotune": {"grouped": [g_lanes, g_slots], "basic": [b_lanes, b_slots]},
        "hit_fraction": hits / nq,
    }
    return sec, tree, keys


def small_section(args, device, bt, flush, stream):
    """The L2-resident basic search: 2^20 unique uniform u32 keys (value =
    rank), 2^20 queries, even slots existing keys, odd slots uniform u32."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    keys, vals, q = wl.point_uniform(1 << 20, 1 << 20)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    dq = torch.from_numpy(q).to(device)
    out = torch.empty(len(q), dtype=torch.uint32, device=device)
    at = importlib.import_module(PKG + ".autotune")
    lanes, rounds, _ = at.tune(tree, dq, mode="basic", repeats=3)
    ms = _timed_ms(lambda: tree.point_search(dq, mode="basic", out=out, stream=stream), stream,
                   flush, max(5, args.steps))
    res = out.cpu().numpy()
    from oracle.oracle import Oracle
    ok = bool(np.array_equal(res, Oracle().point_search(keys, vals, q)))
    tree.close()
    return {"workload": "2^20 unique uniform u32 keys (value = rank), 2^20 queries: 50% keys, "
                        "50% uniform u32; basic search; L2 flushed before every step",
            "value": len(q) / (ms / 1e3), "unit": "queries/s", "ms": ms,
            "lanes_per_query": lanes, "rounds": rounds, "equals_oracle": ok}


def reference_gpu_section(args):
    """The reference's own kernels on this GPU (its .cu sources compiled for
    sm_100a into oracle/_ref/libbtref.so, launched with its wrappers' launch
    shapes; kernel time only, median of 5 after one warm-up).  Keys are padded
    with keys above the largest to a multiple of 5000 (the reference's last
    leaf is always full, main.cu:126-129); the grouped kernel runs with value
    = key (its leaf compares data[], BPTreeExactSearch.cu:269-276)."""
    from oracle.oracle import REF_LIB, RefHarness
    if not os.path.exists(REF_LIB):
        return {"unavailable": "oracle/_ref/libbtref.so not built"}
    wl = importlib.import_module(PKG + ".workloads")
    h = RefHarness()

    def pad(keys):
        keys = keys.astype(np.uint64)
        extra = (-len(keys)) % 5000
        return np.concatenate([keys, keys[-1] + 1 + np.arange(extra, dtype=np.uint64)])

    def med(fn, reps=5):
        fn()
        ts = []
        for _ in range(reps):
            fn()
            ts.append(h.last_ms)
        return statistics.median(ts)

    res = {}
    try:
        keys, vals, q = wl.point_uniform(1 << 20, 1 << 20)
        k = pad(keys)
        h.build(k, np.arange(len(k), dtype=np.uint64))
        ms = med(lambda: h.point_basic(q))
        res["small_basic"] = {"kernel": "kernelSearchingNaiveOneStep (BPTreeExactSearch.cu:25)",
                              "queries": len(q), "ms": ms, "queries_per_s": len(q) / (ms / 1e3)}
        keys, vals, q = zipf_workload(args.grouped_keys_log2, args.queries_log2, 0)
        k = pad(keys)
        h.build(k, np.arange(len(k), dtype=np.uint64))
        ms = med(lambda: h.point_basic(q))
        res["grouped_config_basic"] = {
            "kernel": "kernelSearchingNaiveOneStep (BPTreeExactSearch.cu:25)",
            "queries": len(q), "ms": ms, "queries_per_s": len(q) / (ms / 1e3)}
        lo, hi = wl.range_queries(keys, 1 << 22, 64)
        ms = med(lambda: h.range_basic(lo, hi))
        res["range_basic"] = {
            "kernel": "kernelSearchingKeyRangeGroupStateTwo x2 + kernelGenerateSearchResult "
                      "(BtreeRangeSearch.cu:215, :297)",
            "ranges": len(lo), "ms": ms, "ranges_per_s": len(lo) / (ms / 1e3)}
        h.build(k, k)  # value = key for the grouped kernel
        qg = q[: 1 << 22]
        ms = med(lambda: h.point_grouped(qg), reps=3)
        res["grouped_config_grouped"] = {
            "kernel": "kernelSearchingKeyGroupTwoStep (BPTreeExactSearch.cu:207), kernel only "
                      "(its grouping runs on the host)",
            "queries": len(qg), "ms": ms, "queries_per_s": len(qg) / (ms / 1e3)}
        keys, vals, q = lognormal_workload(args.keys_log2, args.queries_log2, 0)
        k = pad(keys)
        h.build(k, np.arange(len(k), dtype=np.uint64))
        ms = med(lambda: h.point_basic(q))
        res["learned_config_basic"] = {
            "kernel": "kernelSearchingNaiveOneStep (BPTreeExactSearch.cu:25)",
            "queries": len(q), "ms": ms, "queries_per_s": len(q) / (ms / 1e3)}
    finally:
        h.free()
    return res


# ------------------------------------------------------------ GPU leg -------

def run_ours(args):
    import torch
    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = init_dist(world, local_rank)
    bt = importlib.import_module(PKG)
    L = bt.lib()
    P = ctypes.c_void_p

    keys, vals, q = lognormal_workload(args.keys_log2, args.queries_log2, rank)
    nq = len(q)
    stream = torch.cuda.current_stream(device)
    sp = P(stream.cuda_stream)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    rep = tree.learned_train(num_segments=1 << args.segments_log2)
    dq = torch.from_numpy(q).to(device)
    out = torch.empty(nq, dtype=torch.uint64, device=device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)

    def search_learned():
        bt._check(L.bt_point_search(tree.handle, 2, P(dq.data_ptr()), nq, P(out.data_ptr()), sp),
                  "learned")

    def search_plain():
        bt._check(L.bt_point_search(tree.handle, 0, P(dq.data_ptr()), nq, P(out.data_ptr()), sp),
                  "plain")

    # clocks are sampled from here (GPU busy with tuning and warm-up) through
    # the end of the timed region
    clocks = ClockSampler(local_rank)
    clocks.start()
    at = importlib.import_module(PKG + ".autotune")
    p_lanes, p_rounds, _ = at.tune(tree, dq, mode="basic", repeats=3)
    _, l_shape, l_tune_ms = at.tune(tree, dq, mode="learned", repeats=3)
    for _ in range(max(args.warmup, 3)):
        search_learned()
    torch.cuda.synchronize(device)
    learned_res = out.cpu().numpy()
    hits = int(np.count_nonzero(learned_res != np.uint64(0xFFFFFFFFFFFFFFFF)))

    # ---- timed region: K learned steps, device time per step ----------------
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    barrier(dist, device)
    torch.cuda.synchronize(device)
    launches0 = L.bt_kernel_launches()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        search_learned()
        ev[i][1].record(stream)
    torch.cuda.synchronize(device)
    launches = L.bt_kernel_launches() - launches0
    barrier(dist, device)
    clk = clocks.stop()
    step_ms = [e[0].elapsed_time(e[1]) for e in ev]
    ms = max_over_ranks(statistics.mean(step_ms), dist, device)
    value = world * nq / (ms / 1000.0)
    extra, fallback = tree.learned_last_stats()
    extra_lines = tree.learned_last_lines()

    # ---- the plain tree search of the same batch ----------------------------
    for _ in range(2):
        search_plain()
    pev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        pev[i][0].record(stream)
        search_plain()
        pev[i][1].record(stream)
    torch.cuda.synchronize(device)
    plain_ms = max_over_ranks(statistics.mean(e[0].elapsed_time(e[1]) for e in pev), dist, device)
    plain_res = out.cpu().numpy()

    # ---- the reference's batched path on the same batch: radix grouping then
    # the grouped search (BT_POINT_GROUPED, the grouping inside the timing) ---
    def search_grouped():
        bt._check(L.bt_point_search(tree.handle, 1, P(dq.data_ptr()), nq, P(out.data_ptr()), sp),
                  "grouped")

    for _ in range(2):
        search_grouped()
    gev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        gev[i][0].record(stream)
        search_grouped()
        gev[i][1].record(stream)
    torch.cuda.synchronize(device)
    grouped_ms = max_over_ranks(statistics.mean(e[0].elapsed_time(e[1]) for e in gev), dist, device)
    grouped_same = bool(np.array_equal(out.cpu().numpy(), plain_res))

    # ---- end to end through the host-buffer C-ABI call ----------------------
    hq = torch.from_numpy(q).pin_memory()
    hout = torch.empty(nq, dtype=torch.uint64).pin_memory()
    hq_p, hout_p = P(hq.data_ptr()), P(hout.data_ptr())
    for _ in range(2):
        bt._check(L.bt_point_search_host(tree.handle, 2, hq_p, nq, hout_p, sp), "e2e")
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        bt._check(L.bt_point_search_host(tree.handle, 2, hq_p, nq, hout_p, sp), "e2e")
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e_t), dist, device)
    e2e_ok = bool(np.array_equal(hout.numpy(), learned_res))

    # ---- roofline of the learned search kernel -----------------------------
    kb = vb = 8
    # per query: key in, value out, the key's 32-byte sector and, on a hit,
    # its value's sector
    alg_bytes = nq * (kb + vb + 32) + hits * 32
    kernel_s = statistics.mean(step_ms) / 1e3  # this GPU's launches
    achieved = alg_bytes / kernel_s / 1e9
    peak, peak_kind = measured_peak()
    leaf_bytes = -(-len(keys) // 4) * 64
    chain = {f"{l}_line": bt.measure_chain(max(rep["index_bytes"], 1 << 20), leaf_bytes, 1 << 24,
                                           128, l, 2) for l in (1, 2)}
    tq = profiled_traffic("learned_kernel_lognormal_k28_q24")

    sections = {}
    if world == 1:
        sections["serving"] = serving_section(args, bt, tree, keys, (p_lanes, p_rounds),
                                              (p_lanes, p_rounds)) if not args.no_serving else None
    tree.close()
    del dq, out
    if world == 1:
        sections["small"] = small_section(args, device, bt, flush, stream)
        if not args.no_grouped:
            g, gtree, gkeys = grouped_section(args, device, bt, flush, stream)
            sections["grouped"] = g
            sections["ranges"] = range_section(args, device, bt, flush, gtree, gkeys)
            gtree.close()
            sections["build"] = build_section(device, bt, gkeys, np.arange(len(gkeys), dtype=np.uint32))
        if not args.no_forest:
            sections["forest"] = forest_section(args, device, bt, flush)
        if not args.no_rect:
            sections["rectangles"] = rect_section(args, device, bt, flush)
        if not args.no_reference_gpu:
            torch.cuda.synchronize(device)
            torch.cuda.empty_cache()
            sections["reference_gpu"] = reference_gpu_section(args)

    line = None
    if rank == 0:
        cpu = None
        checked = None
        if world == 1 and not args.no_cpu_baseline:
            qps_refc, qps_lb, sample, checked = cpu_refc_qps(keys, vals, q, args.cpu_sample_log2,
                                                             learned_res)
            cpu = {"value": qps_refc, "unit": "queries/s", "cores": os.cpu_count(),
                   "kind": "port",
                   "sample": f"{sample} queries of the batch, reference page tree (fanout 5000) "
                             "restated in C, OpenMP all cores",
                   "lower_bound_qps": qps_lb}
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded)", "config": workload_desc(args),
            "e2e": {"value": world * nq / e2e_s, "unit": "queries/s",
                    "h2d_bytes_per_step": nq * kb, "d2h_bytes_per_step": nq * vb,
                    "api": "bt_point_search_host(BT_POINT_LEARNED), pinned host buffers",
                    "matches_device_result": e2e_ok},
            "plain": {"value": world * nq / (plain_ms / 1e3), "unit": "queries/s",
                      "ms_per_step": plain_ms, "lanes_per_query": p_lanes, "rounds": p_rounds,
                      "api": "bt_point_search(BT_POINT_BASIC)"},
            "plain_grouped": {"value": world * nq / (grouped_ms / 1e3), "unit": "queries/s",
                              "ms_per_step": grouped_ms, "equals_plain": grouped_same,
                              "api": "bt_point_search(BT_POINT_GROUPED): radix grouping + grouped "
                                     "search, the grouping timed"},
            "learned_over_plain": plain_ms / ms,
            "learned_over_plain_grouped": grouped_ms / ms,
            "learned_equals_plain": bool(np.array_equal(learned_res, plain_res)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": None if tq is None else tq * nq,
                         "traffic_source": "not measured in this run: ncu DRAM bytes per query "
                                           "of learned_kernel from a 2^24-key capture "
                                           "(profiles/traffic.json, command there) x queries",
                         "kernel": "learned_kernel",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel_ms": statistics.mean(step_ms),
                         "chain_ceiling": {
                             "queries_per_s": chain,
                             "what": "random 128-byte index line(s) from an L2-sized array of "
                                     "the index's size, then one dependent random 128-byte leaf "
                                     "read (btp_measure_chain)",
                             "frac_1_line": nq / kernel_s / chain["1_line"]}},
            "learned_index": {k: rep[k] for k in ("num_segments", "max_error", "eps_max", "eps_mean",
                                                  "root_error", "root_error_initial",
                                                  "root_loss_initial", "root_loss_final",
                                                  "code_lines_mean", "index_bytes",
                                                  "keys_per_unit", "train_ms")},
            "learned_stats": {"extra_unit_reads": extra, "full_descents": fallback,
                              "extra_code_lines": extra_lines},
            "learned_shape": {"shape": l_shape, "autotune_ms": l_tune_ms},
            "cpu_baseline": cpu,
            "cpu_sample_matches_gpu": checked,
            "clocks": clk,
            "gpu_launches": int(launches),
            "hit_fraction": hits / nq,
            **sections,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def learned_kernel_section(args, device, bt, flush, stream):
    """The learned search kernel alone, for profiling: build and train on the
    learned-index workload, then `steps` learned searches (each after an L2
    flush), timed with CUDA events and checked against the plain search."""
    import torch
    L = bt.lib()
    P = ctypes.c_void_p
    keys, vals, q = lognormal_workload(args.keys_log2, args.queries_log2, 0)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    try:
        rep = tree.learned_train(num_segments=1 << args.segments_log2)
        dq = torch.from_numpy(q).to(device)
        out = torch.empty(len(q), dtype=torch.uint64, device=device)
        ref = torch.empty_like(out)
        sp = P(stream.cuda_stream)
        bt._check(L.bt_point_search(tree.handle, 0, P(dq.data_ptr()), len(q), P(ref.data_ptr()), sp),
                  "plain")
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            bt._check(L.bt_point_search(tree.handle, 2, P(dq.data_ptr()), len(q), P(out.data_ptr()),
                                        sp), "learned")
            e1.record(stream)
            torch.cuda.synchronize(device)
            ms.append(e0.elapsed_time(e1))
        extra, fallback = tree.learned_last_stats()
        return {"keys": len(keys), "queries": len(q), "segments": rep["num_segments"],
                "eps_max": rep["eps_max"], "ms": ms, "equals_plain": bool(torch.equal(out, ref)),
                "extra_unit_reads": extra, "full_descents": fallback,
                "extra_code_lines": tree.learned_last_lines()}
    finally:
        tree.close()


def run_only(args):
    import torch
    bt = importlib.import_module(PKG)
    device = torch.device("cuda:0")
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    if args.only == "learned":
        return run_ours(argparse.Namespace(**{**vars(args), "no_serving": True, "no_grouped": True,
                                              "no_forest": True, "no_rect": True,
                                              "no_reference_gpu": True, "no_cpu_baseline": True}))
    if args.only == "learned_kernel":
        sec = learned_kernel_section(args, device, bt, flush, stream)
    elif args.only in ("grouped", "ranges"):
        sec, gtree, gkeys = grouped_section(args, device, bt, flush, stream)
        if args.only == "ranges":
            sec = range_section(args, device, bt, flush, gtree, gkeys)
        gtree.close()
    elif args.only == "small":
        sec = small_section(args, device, bt, flush, stream)
    else:
        sec = {"forest": forest_section, "rect": rect_section}[args.only](args, device, bt, flush)
    print(json.dumps(sec), flush=True)
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.only:
        return run_only(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
