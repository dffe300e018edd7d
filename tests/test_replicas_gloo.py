"""The multi-GPU bench runs replicas (no collective on the data path): each
rank times its own copy of the workload and the job is as fast as its
slowest rank.  Two gloo ranks on the CPU check that the reduction takes the
maximum over ranks and that the whole-job throughput scales with the ranks."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        ms_max = bench.max_over_ranks(ms, dist, torch, "cpu")
        out[rank] = (ms_max, bench.replica_throughput(world, 1.0e9, ms_max))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    import random
    port = 29500 + random.randint(0, 2000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        # a rank still alive after the join hangs: end it before asserting, so
        # that no process keeps the rendezvous port for later tests
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(10)
        assert [p.exitcode for p in procs] == [0, 0]
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    assert res[0][1] == pytest.approx(2 * 1.0e9 / 0.015 / 1e6)
