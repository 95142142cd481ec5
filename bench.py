#!/usr/bin/env python
"""Benchmark of the B200 B+tree engine.

Default workload (one "step" = one radix-grouped batch point search):
2^26 unique uniform u32 keys (value = rank), bulk-built once; a batch of
2^24 point queries, 90% keys drawn with Zipf(0.99) ranks, 10% uniform u32;
queries radix-grouped by their top 8 bits, then searched.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line on rank 0.  `value` is whole-job queries/s with the
queries resident in HBM (device-timed with CUDA events, max over ranks);
`e2e` is the same metric through the host-buffer C-ABI call
bt_point_search_host (H2D of the queries and D2H of the results inside the
timed region).  The path shards as independent replicas (every rank holds the
tree and answers its own batch, no collective on the data path), so N GPUs
report weak scaling.  `--impl reference` times the CPU restatement of the
reference's algorithm (its fanout-5000 page tree, oracle/oracle.c) on the
host cores.
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
    p.add_argument("--keys-log2", type=int, default=26)
    p.add_argument("--queries-log2", type=int, default=24)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-log2", type=int, default=22)
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-index + serving section (2^28 u64 keys)")
    p.add_argument("--learned-keys-log2", type=int, default=28)
    p.add_argument("--serve-requests", type=int, default=3000)
    p.add_argument("--serve-rate", type=float, default=20000.0, help="requests per second")
    p.add_argument("--no-forest", action="store_true", help="skip the 4096-tree forest section")
    p.add_argument("--no-rect", action="store_true", help="skip the rectangle-search section")
    p.add_argument("--rect-boxes-log2", type=int, default=20, help="boxes in the rectangle section")
    p.add_argument("--forest-trees", type=int, default=4096, help="trees in the forest section")
    p.add_argument("--only", choices=["learned", "forest", "rect"],
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

def workload(keys_log2, queries_log2, rank):
    wl = importlib.import_module(PKG + ".workloads")
    cache = os.path.join(tempfile.gettempdir(), "btree_b200_bench")
    os.makedirs(cache, exist_ok=True)
    tag = f"zipf_k{keys_log2}_q{queries_log2}_r{rank}"
    f = os.path.join(cache, tag + ".npz")
    if os.path.exists(f):
        d = np.load(f)
        return d["keys"], d["vals"], d["q"]
    keys, vals, q = wl.point_zipf(1 << keys_log2, 1 << queries_log2, seed=wl.KEY_SEED)
    if rank:
        # each replica answers its own batch (weak scaling)
        _, _, q = wl.point_zipf(1 << keys_log2, 1 << queries_log2, seed=wl.KEY_SEED + 100 * rank)
    np.savez(f, keys=keys, vals=vals, q=q)
    return keys, vals, q


def workload_desc(args):
    return {
        "workload": (f"radix-grouped point search: 2^{args.keys_log2} unique uniform u32 keys "
                     f"(value = rank), batches of 2^{args.queries_log2} queries, 90% keys by "
                     "Zipf(0.99) rank, 10% uniform u32; grouped by the top 8 key bits"),
        "keys": 1 << args.keys_log2,
        "queries_per_step": 1 << args.queries_log2,
        "key_type": "u32", "value_type": "u32",
        "l2": "flushed before every timed step (512 MiB write); tree (512 MiB) > L2",
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
    keys, vals, q = workload(args.keys_log2, args.queries_log2, 0)
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
                                   "tree (fanout 5000) restated in C, OpenMP"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------ learned index + serving --------

def learned_section(args, device, bt, flush):
    """Learned index and serving workload: 2^28 unique u64 keys (cumulative sum of
    floor(lognormal(4, 2)) + 1 gaps), value = rank; FP32 two-stage model with
    2^16 leaf segments trained on the GPU.  Reports the plain and the learned
    batched point-search throughput on a 2^24-query batch (90% hits uniform
    over ranks, 10% uniform in [min, max]) and p50/p99 latency of a Poisson
    request loop with batch sizes round(2^U), U ~ uniform[0, 16]."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    at = importlib.import_module(PKG + ".autotune")
    n = 1 << args.learned_keys_log2
    keys = wl.lognormal_keys(n)
    vals = np.arange(n, dtype=np.uint64)
    g = wl.rng(wl.KEY_SEED + 7)
    nq = 1 << args.queries_log2
    q = keys[g.integers(0, n, size=nq)]
    miss = g.random(nq) < 0.10
    q[miss] = g.integers(int(keys[0]), int(keys[-1]) + 1, size=int(miss.sum()), dtype=np.uint64)
    stream = torch.cuda.current_stream(device)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    rep = tree.learned_train(num_segments=1 << 16, hidden=16, iterations=400)
    dq = torch.from_numpy(q).to(device)
    out = torch.empty(nq, dtype=torch.uint64, device=device)

    def timed(fn, steps):
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

    lanes_p, rounds_p, _ = at.tune(tree, dq, mode="basic", repeats=3)
    plain_ms = timed(lambda: tree.point_search(dq, mode="basic", out=out, stream=stream), args.steps)
    plain_res = out.cpu().numpy()
    learned_ms = {}
    for cfg in tree.SEARCH_CONFIGS:  # the autotuner's choice for the learned kernel
        tree.set_search_config(*cfg)
        learned_ms[cfg] = timed(lambda: tree.point_search_learned(dq, out=out, stream=stream), 2)
    best = min(learned_ms, key=learned_ms.get)
    tree.set_search_config(*best)
    l_ms = timed(lambda: tree.point_search_learned(dq, out=out, stream=stream), args.steps)
    learned_res = out.cpu().numpy()
    windowed, fallback = tree.learned_last_stats()
    hits = int(np.count_nonzero(learned_res != np.uint64(0xFFFFFFFFFFFFFFFF)))
    exact = bool(np.array_equal(learned_res, plain_res))
    alg = nq * (8 + 8 + 32) + hits * 32
    peak, _ = measured_peak()

    # request loop: Poisson arrivals, log-uniform batch sizes, pinned buffers
    sizes = np.rint(2.0 ** g.uniform(0, 16, size=args.serve_requests)).astype(np.int64)
    reqs = []
    for m in sizes:
        r = keys[g.integers(0, n, size=m)]
        mm = g.random(m) < 0.10
        r[mm] = g.integers(int(keys[0]), int(keys[-1]) + 1, size=int(mm.sum()), dtype=np.uint64)
        reqs.append(torch.from_numpy(r).pin_memory().numpy())
    outs = [torch.empty(len(r), dtype=torch.uint64).pin_memory().numpy() for r in reqs]
    arrivals = np.cumsum(g.exponential(1e6 / args.serve_rate, size=len(reqs)))
    serving = {}
    for mode in ("basic", "learned"):
        tree.set_search_config(*(best if mode == "learned" else (lanes_p, rounds_p)))
        with bt.Server(tree, mode=mode, slots=8, memory_budget_bytes=512 << 20) as srv:
            srv.replay(reqs[:200], arrivals[:200] - arrivals[0], outs[:200])  # warm-up
            lat, wall, _ = srv.replay(reqs, arrivals - arrivals[0], outs)
            st = srv.stats()
        serving[mode] = {"p50_us": float(np.percentile(lat, 50)),
                         "p99_us": float(np.percentile(lat, 99)),
                         "mean_us": float(lat.mean()),
                         "queries_per_s": float(sizes.sum() / (wall / 1e6)),
                         "max_in_flight": st["max_in_flight"], "slots": st["slots"]}
    tree.close()
    return {
        "workload": (f"2^{args.learned_keys_log2} unique u64 keys = cumsum(floor(lognormal(4,2))+1), "
                     f"value = rank; batch of 2^{args.queries_log2} queries, 90% hits uniform over "
                     "ranks, 10% uniform in [min, max]"),
        "plain": {"value": nq / (plain_ms / 1e3), "unit": "queries/s", "ms": plain_ms,
                  "lanes_per_query": lanes_p, "rounds": rounds_p},
        "learned": {"value": nq / (l_ms / 1e3), "unit": "queries/s", "ms": l_ms,
                    "lanes_per_query": best[0], "rounds": best[1],
                    "windowed": windowed, "fallback": fallback,
                    "roofline": {"bound": "hbm", "achieved": alg / (l_ms / 1e3) / 1e9,
                                 "peak": peak, "unit": "GB/s",
                                 "frac": alg / (l_ms / 1e3) / 1e9 / peak}},
        "learned_over_plain": plain_ms / l_ms,
        "exact": exact,
        "model": {k: rep[k] for k in ("root_loss_initial", "root_loss_final", "eps_mean",
                                      "eps_max", "window_lines_mean", "train_ms",
                                      "keys_per_entry")},
        "serving": {"requests": int(len(reqs)), "rate_per_s": args.serve_rate,
                    "batch_sizes": "round(2^U), U ~ uniform[0,16]", **serving},
    }


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
    captured CUDA graph.  The plan's lanes/rounds and tile are chosen by
    timing the candidates."""
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    keys, vals, koff, q, qoff, lo, hi, roff = wl.forest(num_trees=args.forest_trees)
    stream = torch.cuda.current_stream(device)
    f = bt.Forest(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device), koff)
    dq = torch.from_numpy(q).to(device)
    dlo, dhi = torch.from_numpy(lo).to(device), torch.from_numpy(hi).to(device)
    out = torch.empty(len(q), dtype=torch.uint32, device=device)
    counts = torch.empty(len(lo), dtype=torch.uint64, device=device)
    tried = {}
    for cfg in ((4, 1), (8, 1), (8, 2)):
        for tile in (512, 2048, 8192):
            with f.plan(dq, qoff, out, dlo, dhi, roff, counts, *cfg, tile=tile) as p:
                p.run(stream)
                tried[f"{cfg[0]}x{cfg[1]}/t{tile}"] = _timed_ms(lambda: p.run(stream), stream, flush, 3)
    best = min(tried, key=tried.get)
    lanes, rounds = (int(x) for x in best.split("/")[0].split("x"))
    tile = int(best.split("/t")[1])
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
        "tile": tile, "autotune_ms": tried, "answers_consistent": ok,
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
    return {"keys": len(keys), "sorted_ms": sorted_ms, "unsorted_ms": unsorted_ms,
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
        "ids": {"ranges_per_s": nr / (ms_ids / 1e3), "ms": ms_ids, "hits": hits,
                "api": "Tree.range_search (counts, scan, offsets, ID fill)"},
        "roofline": {"bound": "hbm", "kernel": "bounds_kernel (basic counts)",
                     "achieved": alg / (base_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (base_ms / 1e3) / 1e9 / peak},
    }


def rect_section(args, device, bt, flush):
    """Rectangle workload: 2^24 points (x, y uniform u16) keyed by their
    32-bit Morton code (value = point ID, sorted by (code, ID)); 2^20
    rectangles with a uniform corner and sides uniform in [1, 256].  Timed:
    one bt_rect_search call (count pass, scan, fill pass, per-box ID sort)
    into a buffer sized by an untimed first call; beside it the reference's
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
    cargs = (tree.handle, *(P(t.data_ptr()) for t in d), len(x0), P(counts.data_ptr()),
             P(offsets.data_ptr()), P(hits.data_ptr()), len(hits), ctypes.byref(total),
             P(stream.cuda_stream))

    def run():
        st = bt.lib().bt_rect_search(*cargs)
        if st != 0:
            raise RuntimeError(f"bt_rect_search failed with status {st}")

    l0 = bt.kernel_launches()
    ms = _timed_ms(run, stream, flush, max(3, args.steps // 3))
    launches = (bt.kernel_launches() - l0) / max(3, args.steps // 3)
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
        "hits": nh, "hits_per_rect": nh / len(x0), "answers_consistent_first_2048": ok,
        "z_interval_counts": zi,
        "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak},
    }


# ------------------------------------------------------------ GPU leg -------

def run_ours(args):
    import torch
    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = init_dist(world, local_rank)
    bt = importlib.import_module(PKG)
    L = bt.lib()

    keys, vals, q = workload(args.keys_log2, args.queries_log2, rank)
    nq = len(q)
    stream = torch.cuda.current_stream(device)
    tree = bt.Tree.build(torch.from_numpy(keys).to(device), torch.from_numpy(vals).to(device))
    dq = torch.from_numpy(q).to(device)
    grouped = torch.empty_like(dq)
    perm = torch.empty(nq, dtype=torch.uint32, device=device)
    out = torch.empty(nq, dtype=torch.uint32, device=device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)

    P = ctypes.c_void_p
    sp = P(stream.cuda_stream)

    def group_into():
        bt._check(L.bt_group_queries(tree.handle, P(dq.data_ptr()), nq, P(grouped.data_ptr()),
                                     P(perm.data_ptr()), sp), "group")

    def search_grouped():
        bt._check(L.bt_point_search_grouped_batch(tree.handle, P(grouped.data_ptr()),
                                                  P(perm.data_ptr()), nq, P(out.data_ptr()), sp),
                  "search")

    def search_basic():
        bt._check(L.bt_point_search(tree.handle, 0, P(dq.data_ptr()), nq, P(out.data_ptr()), sp),
                  "basic")

    # clocks are sampled from here (GPU busy with tuning and warm-up) through
    # the end of the timed region, which alone is shorter than one sample
    clocks = ClockSampler(local_rank)
    clocks.start()
    # the project's autotuner picks the kernel shape per mode (untimed)
    at = importlib.import_module(PKG + ".autotune")
    b_lanes, b_slots, b_ms = at.tune(tree, dq, mode="basic", repeats=3)
    g_lanes, g_slots, g_ms = at.tune(tree, dq, mode="grouped", repeats=3)

    # warm-up (the result is compared with the CPU leg's sample on rank 0)
    for _ in range(max(args.warmup, 3)):
        group_into()
        search_grouped()
    torch.cuda.synchronize(device)
    res = out.cpu().numpy()
    hits = int(np.count_nonzero(res != np.uint32(0xFFFFFFFF)))
    checked = None

    # ---- timed region: K grouped steps, device time per step ----------------
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    barrier(dist, device)
    torch.cuda.synchronize(device)
    launches0 = L.bt_kernel_launches()
    nvtx = torch.cuda.nvtx
    for i in range(args.steps):
        flush.zero_()
        nvtx.range_push("timed_grouped")
        ev[i][0].record(stream)
        group_into()
        ev[i][1].record(stream)
        search_grouped()
        ev[i][2].record(stream)
        nvtx.range_pop()
    torch.cuda.synchronize(device)
    launches = L.bt_kernel_launches() - launches0
    barrier(dist, device)
    clk = clocks.stop()
    step_ms = [ev[i][0].elapsed_time(ev[i][2]) for i in range(args.steps)]
    search_ms = [ev[i][1].elapsed_time(ev[i][2]) for i in range(args.steps)]
    group_ms = [ev[i][0].elapsed_time(ev[i][1]) for i in range(args.steps)]
    ms = max_over_ranks(statistics.mean(step_ms), dist, device)
    value = world * nq / (ms / 1000.0)

    # ---- ungrouped basic search, same batch (the plain path) ----------------
    tree.set_search_config(b_lanes, b_slots)
    for _ in range(2):
        search_basic()
    bev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        nvtx.range_push("timed_basic")
        bev[i][0].record(stream)
        search_basic()
        bev[i][1].record(stream)
        nvtx.range_pop()
    torch.cuda.synchronize(device)
    basic_ms = max_over_ranks(statistics.mean(b[0].elapsed_time(b[1]) for b in bev), dist, device)

    # ---- end to end through the host-buffer C-ABI call ----------------------
    tree.set_search_config(g_lanes, g_slots)
    hq = torch.from_numpy(q).pin_memory()
    hout = torch.empty(nq, dtype=torch.uint32).pin_memory()
    hq_p, hout_p = P(hq.data_ptr()), P(hout.data_ptr())
    for _ in range(2):
        bt._check(L.bt_point_search_host(tree.handle, 1, hq_p, nq, hout_p, sp), "e2e")
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        bt._check(L.bt_point_search_host(tree.handle, 1, hq_p, nq, hout_p, sp), "e2e")
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e_t), dist, device)
    e2e_ok = bool(np.array_equal(hout.numpy(), res))

    # ---- roofline of the dominant kernel (the grouped search kernel) --------
    kb = vb = 4
    # per launch: key in, value out, the leaf block's key sector, and its
    # value sector on a hit
    alg_bytes = nq * (kb + vb + 32) + hits * 32
    search_s = statistics.mean(search_ms) / 1000.0
    achieved = alg_bytes / search_s / 1e9
    peak, peak_kind = measured_peak()
    # the ceiling for one random leaf-block read per query: random 64-byte
    # reads over a region the size of the tree's leaves, measured here
    leaf_bytes = -(-len(keys) // (32 // kb)) * 64
    gather_rps = bt.measure_gather(leaf_bytes, 1 << 24, 64)
    tq = profiled_traffic("point_kernel_grouped_zipf_k26_q24")

    ranges = range_section(args, device, bt, flush, tree, keys) if world == 1 else None
    build = build_section(device, bt, keys, vals) if world == 1 else None
    learned = forest = rect = None
    if world == 1 and not args.no_learned:
        learned = learned_section(args, device, bt, flush)
    if world == 1 and not args.no_forest:
        forest = forest_section(args, device, bt, flush)
    if world == 1 and not args.no_rect:
        rect = rect_section(args, device, bt, flush)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            qps_refc, qps_lb, sample, checked = cpu_refc_qps(keys, vals, q, args.cpu_sample_log2, res)
            cpu = {"value": qps_refc, "unit": "queries/s", "cores": os.cpu_count(),
                   "kind": "port",
                   "sample": f"{sample} queries of the batch, reference page tree (fanout 5000) "
                             "restated in C, OpenMP all cores",
                   "lower_bound_qps": qps_lb}
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)", "config": workload_desc(args),
            "e2e": {"value": world * nq / e2e_s, "unit": "queries/s",
                    "h2d_bytes_per_step": nq * kb, "d2h_bytes_per_step": nq * vb,
                    "api": "bt_point_search_host (grouped), pinned host buffers",
                    "matches_device_result": e2e_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": None if tq is None else tq * nq,
                         "kernel": "point_window_kernel (grouped batch)",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel_ms": statistics.mean(search_ms),
                         "random_gather_ceiling": {
                             "reads_per_s": gather_rps, "block_bytes": 64,
                             "region_bytes": leaf_bytes,
                             "search_queries_per_s": nq / search_s,
                             "frac": nq / search_s / gather_rps}},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches),
            "breakdown_ms": {"group": statistics.mean(group_ms),
                             "search": statistics.mean(search_ms)},
            "plain_basic": {"value": world * nq / (basic_ms / 1000.0), "unit": "queries/s",
                            "ms_per_step": basic_ms},
            "hit_fraction": hits / nq,
            "autotune": {"grouped": {"lanes_per_query": g_lanes, "queries_per_group": g_slots,
                                     "ms": g_ms},
                         "basic": {"lanes_per_query": b_lanes, "queries_per_group": b_slots,
                                   "ms": b_ms}},
            "cpu_sample_matches_gpu": checked,
            "learned_index": learned,
            "forest": forest,
            "rectangles": rect,
            "ranges": ranges,
            "build": build,
        }
        print(json.dumps(line), flush=True)
    tree.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_only(args):
    import torch
    bt = importlib.import_module(PKG)
    device = torch.device("cuda:0")
    torch.cuda.set_device(device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    fn = {"learned": learned_section, "forest": forest_section, "rect": rect_section}[args.only]
    print(json.dumps(fn(args, device, bt, flush)), flush=True)
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
