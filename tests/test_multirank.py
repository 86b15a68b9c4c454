"""The multi-GPU host logic of bench.py on CPU ranks (gloo, world size 2): the
step time is the maximum over ranks, the value aggregates all ranks' work, and
every rank draws its own phantom (independent scans, weak scaling)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import bench
    from analyticalreconbigpatient_b200 import geometry as G, phantom as P

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dev = torch.device("cpu")
        times = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 0.25 * (rank + 1)], world, dev)
        sc = G.config("small")
        objs = P.random_ellipsoids(1000 + rank, 8, (-10.0, 10.0))
        # every rank agrees on the aggregate; phantoms differ between ranks
        digest = torch.tensor([float(np.abs(objs).sum())], dtype=torch.float64)
        gathered = [torch.zeros_like(digest) for _ in range(world)]
        dist.all_gather(gathered, digest)
        out.put((rank, times, bench.job_gups(sc.updates(), world, times[0]), [float(g) for g in gathered]))
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_reduce_times_and_draw_their_own_phantoms():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        rank, times, gups, digests = q.get(timeout=120)
        res[rank] = (times, gups, digests)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from analyticalreconbigpatient_b200 import geometry as G

    for rank in (0, 1):
        times, gups, digests = res[rank]
        assert times == [2.0, 5.0, 0.5]
        assert gups == pytest.approx(G.config("small").updates() * 2 / 2.0 / 1e9)
        assert digests[0] != digests[1]


def test_single_process_is_unchanged():
    import bench

    assert bench.max_over_ranks([3, 1.5], 1, None) == [3.0, 1.5]
