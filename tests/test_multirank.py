"""The replica path of `bench.py` under two ranks on CPU (gloo): disjoint
atmosphere seeds per rank, the max over ranks of the device time, and the
whole-job value computed from the slowest rank. No GPU is involved."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        seeds = bench.rank_seeds(4, rank)
        ms_local = 10.0 + 5.0 * rank            # rank 1 is the slower one
        ms = bench.max_over_ranks(ms_local, dist, world, "cpu")
        out.put((rank, seeds, ms, bench.job_value(world, 4, ms)))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, ms0, v0), (r1, s1, ms1, v1) = res
    assert not set(s0) & set(s1)                 # disjoint atmospheres
    assert ms0 == ms1 == 15.0                    # both see the slowest rank's time
    assert v0 == v1 == pytest.approx(2 * 4 / 15e-3)
