"""CPU: the multi-rank plumbing of bench.py with two gloo processes.

`bench.py --gpus N` runs one process per GPU; every rank takes its own shard
of the workload (its own seeded rays, frame or batch of scenes: weak scaling,
no exchange on the data path), the timed region is bracketed by barriers and
the job's rate is the units of all ranks over the slowest rank's time.  Here
the same functions run in two CPU processes over gloo (DORT_DIST_BACKEND),
rendezvous on 127.0.0.1.
"""
from __future__ import annotations

import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), DORT_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    from dort_b200 import scenes
    r, w, _, pg = bench.dist_setup(world)
    assert (r, w) == (rank, world) and pg is not None
    bench.barrier(pg)
    seconds = 1.0 + rank                      # this rank's timed region
    slowest = bench.max_over_ranks(pg, seconds)
    rate = bench.job_rate(100.0, w, slowest)
    seeds = [None] * w
    pg.all_gather_object(seeds, bench.rank_seed(42, rank))
    jobs = scenes.batch_jobs(count=2, seed=bench.rank_seed(4, rank), min_tris=1000,
                             max_tris=2000)
    shard = [(len(j[0]["tris"]), j[1], j[2], j[3], j[4]) for j in jobs]
    shards = [None] * w
    pg.all_gather_object(shards, shard)
    bench.barrier(pg)
    pg.destroy_process_group()
    out.put((rank, slowest, rate, seeds, shards))


def test_two_gloo_ranks_shard_time_and_aggregate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, slowest, rate, seeds, shards in results:
        assert slowest == 2.0                  # the max over ranks, on every rank
        assert rate == pytest.approx(100.0)    # 2 ranks x 100 units / 2 s
        assert seeds[0] != seeds[1]            # independent shards
        assert shards[0] != shards[1]
    assert results[0][3] == results[1][3] and results[0][4] == results[1][4]
