"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The search path shards as independent replicas: every rank builds its own
tree and answers its own batch, with no collective on the data path.  The
only cross-rank steps are the barrier around the timed region and the
max-over-ranks reduction of the step time; both are checked here with gloo.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    r, w, lr = bench.dist_env()
    assert (r, w, lr) == (rank, world, rank)
    dist = bench.init_dist(w, lr, backend="gloo")
    try:
        bench.barrier(dist)
        mine = 1.5 + rank          # this rank's mean step time (ms)
        slowest = bench.max_over_ranks(mine, dist)
        q.put((rank, slowest))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert got == [(0, 2.5), (1, 2.5)]


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.init_dist(1, 0) is None
    assert bench.max_over_ranks(3.0, None) == 3.0


@pytest.mark.parametrize("rank", [0, 1, 3])
@pytest.mark.parametrize("which", ["lognormal_workload", "zipf_workload"])
def test_replica_batches_differ_per_rank(rank, which, monkeypatch, tmp_path):
    """Weak scaling: each rank answers its own batch over the same keys."""
    import bench
    monkeypatch.setattr(bench.tempfile, "gettempdir", lambda: str(tmp_path))
    make = getattr(bench, which)
    k0, v0, q0 = make(12, 10, 0)
    k, v, q = make(12, 10, rank)
    assert (k == k0).all() and (v == v0).all()
    assert (q == q0).all() == (rank == 0)
