"""The multi-rank logic of bench.py (one replica workload per GPU, the job's
value = all ranks' terms / the slowest rank's time) on CPU `gloo` ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    maxes, sums = bench.combine_ranks(torch, dist, "cpu", [10.0 + rank, 3.0 - rank, 0.5],
                                      [1000 + rank, 7, 2 ** 40])
    out[rank] = (maxes, sums)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_combine_ranks_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        maxes, sums = res[r]
        assert maxes == [10.0 + world - 1, 3.0, 0.5]
        assert sums == [1000 * world + sum(range(world)), 7 * world, float(2 ** 40 * world)]



def test_combine_ranks_single():
    import torch

    import bench
    assert bench.combine_ranks(torch, None, "cpu", [1.5], [3]) == ([1.5], [3])
