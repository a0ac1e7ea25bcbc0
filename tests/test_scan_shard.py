"""A scan split across ranks (gloo, two processes on the CPU): each point is solved by
exactly one rank, the shares balance by cost, and rank 0 reassembles the results."""

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from solprop_b200 import scan


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        points = scan.draw_points(37, 5)
        mine = scan.shard(points, rank, world)
        # a stand-in for each run's exit spectrum: a function of the point alone
        values = np.array([[p.radius, p.energy, p.n_to] for p in (points[i] for i in mine)])
        full = scan.gather_by_index(mine, values, len(points))
        if rank == 0:
            out.put(("full", full))
        out.put(("cost", rank, sum(points[i].n_to * points[i].modes for i in mine)))
    finally:
        dist.destroy_process_group()


def test_shards_cover_the_scan_once_and_balance():
    points = scan.draw_points(37, 5)
    shards = [scan.shard(points, r, 3) for r in range(3)]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(37))
    costs = [sum(points[i].n_to * points[i].modes for i in s) for s in shards]
    assert max(costs) - min(costs) <= max(p.n_to * p.modes for p in points)


def test_two_gloo_ranks_gather_every_point_on_rank_0():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msgs = [q.get(timeout=120) for _ in range(3)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = next(m[1] for m in msgs if m[0] == "full")
    points = scan.draw_points(37, 5)
    expect = np.array([[p.radius, p.energy, p.n_to] for p in points])
    assert np.array_equal(full, expect)
    costs = sorted(m[2] for m in msgs if m[0] == "cost")
    assert len(costs) == 2 and costs[1] - costs[0] <= max(p.n_to * p.modes for p in points)
