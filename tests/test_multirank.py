"""The replicas path of `bench.py --gpus N` on CPU ranks (gloo, world size 2, spawned processes):
each rank draws its own disjoint pairs, the step time is the maximum over ranks, and the whole-job
rate counts every rank's pairs over that time. The pairs are independent units, so the path has
no data-path collective; only the timing reduction crosses ranks."""
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s0 = bench.rank_seed(1000, rank)
        seeds = list(range(s0, s0 + 64))      # gen_pairs(64, s0) draws pairs with these seeds
        every = [None] * world
        dist.all_gather_object(every, seeds)
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        q.put((rank, every, ms, bench.job_rate(world, 64, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, every, ms, rate in res:
        assert set(every[0]).isdisjoint(every[1])
        assert ms == 15.0                        # the slower rank's time, on both ranks
        assert rate == pytest.approx(2 * 64 / 0.015)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(12.5, None, None) == 12.5
    assert bench.rank_seed(1000, 0) == 1000
    assert bench.job_rate(1, 64, 150.0) == pytest.approx(64 / 0.150)
