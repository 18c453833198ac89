"""The bench's multi-rank logic on CPU (gloo, world size 2): replicas seeded
by rank, barriers around the timed region, the job's time = the max over
ranks, and rank 0 alone reporting."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist

    r, w, local, pg = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(pg)
        # each rank's "time": the slowest rank decides the job's time
        t = bench.dist_max(10.0 + 5.0 * r, pg)
        from andosim_b200 import scenes

        sc = scenes.c4(seed=r, n=8)  # replicas are seeded by rank
        first = float(sc.vertices[0, 0])
        bench.barrier(pg)
        out.put((r, w, t, first))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_and_differ_in_seed():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r for r, *_ in res] == [0, 1] and all(w == 2 for _, w, _, _ in res)
    assert all(t == 15.0 for _, _, t, _ in res)          # max over ranks on every rank
    assert res[0][3] != res[1][3]                          # different replicas


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r, w, local, pg = bench.dist_setup(1)
    assert (r, w, local, pg) == (0, 1, 0, False)
    assert bench.dist_max(3.5, pg) == 3.5
