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


def test_lpt_partition():
    from srg_b200 import partition as PT
    w = [5, 9, 9, 1, 7, 3, 3]
    parts = PT.lpt_partition(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(w)))
    assert all(p == sorted(p) for p in parts)
    loads = [sum(w[i] for i in p) for p in parts]
    # LPT: 9, 9, 7 to ranks 0, 1, 2; then 5 -> 2, 3 -> 0, 3 -> 1, 1 -> 0
    assert parts == [[1, 3, 5], [2, 6], [0, 4]] and loads == [13, 12, 12]
    assert PT.lpt_partition(w, 1) == [list(range(len(w)))]
    assert PT.owners(parts, len(w)) == [2, 0, 1, 0, 2, 0, 1]
    # more ranks than bursts: the extra ranks get nothing
    assert PT.lpt_partition([1, 1], 4) == [[0], [1], [], []]


def _scene_bursts():
    """Six bursts on one grid whose boxes overlap (the mini scene's three
    bursts, then the same geometry with other samples)."""
    import copy

    from srg_b200 import scene
    grid, bursts = scene.mini_scene()
    more = []
    for i, b in enumerate(bursts):
        c = copy.copy(b)
        c.burst = scene.mini_samples(900 + i, b.burst.shape[0], b.burst.shape[1])
        more.append(c)
    return grid, bursts + more


def _images(bursts, idx):
    """Oracle images (GPU form) of the bursts in idx, each cropped to its box
    [firstpix, min(lastpix, W-1)] as the device layout holds it."""
    import numpy as np
    import torch

    import oracle as O
    from srg_b200 import api
    orc = O.Oracle()
    out = {}
    for i in idx:
        b = bursts[i]
        fl, ll, fp, lp = api.limits(b)
        img = orc.stages(b, gpu_lerp=1, gpu_scale=1, nthreads=1)["out"]
        out[i] = torch.from_numpy(np.ascontiguousarray(img[:, fp:min(lp, b.demwidth - 1) + 1]))
    return out


def _merge(raster, bursts, images):
    """The reference's ordered merge (|Re| > 1e-18 replaces), burst by burst."""
    from srg_b200 import api
    for i, b in enumerate(bursts):
        fl, ll, fp, lp = api.limits(b)
        img = images[i]
        box = raster[fl:fl + img.shape[0], fp:fp + img.shape[1]]
        box[:] = img.where(img.real.abs() > 1e-18, box)
    return raster


def _partition_worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from srg_b200 import partition as PT
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    grid, bursts = _scene_bursts()
    n = len(bursts)
    weights = [b.rawdatalines * b.samples for b in bursts]   # any deterministic estimate
    parts = PT.lpt_partition(weights, world)
    own = PT.owners(parts, n)
    mine = _images(bursts, parts[rank])
    # every rank holds a buffer per burst; only its own are filled
    shapes = {i: v.shape for i, v in _images(bursts, range(n)).items()} if rank == 0 else None
    outs = []
    for i in range(n):
        if i in mine:
            outs.append(mine[i])
        elif rank == 0:
            outs.append(torch.zeros(shapes[i], dtype=torch.complex64))
        else:
            outs.append(None)
    PT.gather_outputs(outs, own, rank, dist)
    if rank == 0:
        raster = torch.zeros((grid.length, grid.width), dtype=torch.complex64)
        got = _merge(raster, bursts, outs)
        out["got"] = got.numpy().copy()
        out["parts"] = parts
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_scene_merges_like_one_rank_gloo(world):
    """Bursts dealt by LPT over `world` gloo ranks, each rank forming only its
    own bursts' images, gathered to rank 0 and merged there in burst order:
    the raster is bit-identical to one rank merging every image in order."""
    import numpy as np
    import torch
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_partition_worker, args=(r, world, port, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        got, parts = out["got"], out["parts"]
    assert all(len(p) > 0 for p in parts) and len(parts) == world
    grid, bursts = _scene_bursts()
    ref = _merge(torch.zeros((grid.length, grid.width), dtype=torch.complex64), bursts,
                 _images(bursts, range(len(bursts)))).numpy()
    assert np.count_nonzero(ref) > 0
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_block_partition():
    from srg_b200 import partition
    assert partition.block_partition(32, 3) == [list(range(0, 11)), list(range(11, 22)),
                                                list(range(22, 32))]
    assert partition.block_partition(32, 8) == [list(range(4 * k, 4 * k + 4)) for k in range(8)]
    assert partition.block_partition(5, 1) == [[0, 1, 2, 3, 4]]
    for n in range(1, 40):
        for w in range(1, 9):
            parts = partition.block_partition(n, w)
            assert sum(parts, []) == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition.block_partition(4, 0)


def _pairs(images):
    """A stand-in for the interferograms of sequential pairs (k, k+1)."""
    import torch
    return [torch.conj(images[k]) * images[k + 1] for k in range(len(images) - 1)]


def _stack_worker(rank, world, port, n, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from srg_b200 import partition
    g = torch.Generator().manual_seed(11)
    every = [torch.complex(torch.randn(6, 5, generator=g), torch.randn(6, 5, generator=g))
             for _ in range(n)]
    block = partition.block_partition(n, world)[rank]
    mine = [every[i].clone() for i in block]
    recv = torch.empty_like(mine[0])
    nxt = partition.exchange_boundary(mine[0], recv, rank, world, dist)
    imgs = mine + ([nxt] if nxt is not None else [])
    pairs = _pairs(imgs)
    out[rank] = (block[0], [p.numpy() for p in pairs])
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_stack_blocks_with_boundary_exchange_give_every_pair_gloo(world):
    """A 7-image stack dealt in date-order blocks over `world` gloo ranks: with
    the one exchange per block boundary the ranks' sequential pairs are, in
    order, exactly the one-rank stack's 6 pairs, bit for bit."""
    import numpy as np
    import torch
    import torch.multiprocessing as mp
    n = 7
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_stack_worker, args=(r, world, port, n, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    got = []
    for r in range(world):
        first, pairs = res[r]
        got += pairs
    g = torch.Generator().manual_seed(11)
    every = [torch.complex(torch.randn(6, 5, generator=g), torch.randn(6, 5, generator=g))
             for _ in range(n)]
    want = [p.numpy() for p in _pairs(every)]
    assert len(got) == n - 1
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
