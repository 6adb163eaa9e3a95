"""The multi-rank host logic of bench.py on CPU: two gloo ranks.

Each rank propagates its own seeded source points (replicas, no collective in
the data path); the only collective is the maximum of the ranks' device times.
"""

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]
    import bench
    from workloads import light_run

    dist, r, ws, local = bench._dist(backend="gloo")
    assert (r, ws) == (rank, world)
    run = light_run()
    pts = bench.rank_points(run, 4, r, (0.1, 0.3))
    t = bench._max_over_ranks(dist, local, [1.0 + r, 5.0 - r])
    out.put((r, [p["gamma"] for p in pts], t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_points_and_reduce_the_maximum():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, g0, t0), (r1, g1, t1) = res
    assert g0 != g1                 # each rank draws its own points
    assert t0 == t1 == [2.0, 5.0]   # both ranks see the maximum of each time


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path[:0] = [ROOT]
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"points": 4, "z_range": (0.1, 0.2), "warmup": 0, "steps": 1})()
    assert bench.reference_arm(args) is None
    assert capsys.readouterr().out == ""
