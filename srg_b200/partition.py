"""A scene's bursts shared among ranks (one process per GPU), and the ordered
gather of their images.

Each output pixel depends on its own burst's pulses only, so the bursts of a
scene are independent units, with no reduction between them.  The reference
processes a scene's bursts one after another and merges each into the .geo
raster in that order, a later burst replacing an earlier one where both form
a pixel (sentinel/backprojectgpusub.f90:140-248 calling azimuth_compress_,
whose merge is azimuth_compress.cu:510-537).  Here:

* ``lpt_partition`` deals the bursts to ranks by estimated work (executed
  terms), longest first, each to the least-loaded rank (the LPT rule); each
  rank then backprojects its bursts in one persistent launch;
* ``gather_outputs`` sends every burst image to the merging rank with
  point-to-point operations (NCCL between GPUs, gloo between CPU ranks):
  only the burst boxes cross the links, never a full raster, and remote data
  land in local memory before any kernel reads them;
* the merging rank merges the images into the raster in global burst order
  (``ordered_merge``), which reproduces the one-rank result bit for bit: a
  pixel ends with the image of the last burst that replaced it, whichever
  rank computed that image.

A repeat-pass stack (acquisitions of one footprint, interferograms of the
sequential pairs) is dealt in contiguous blocks of the date order instead
(``block_partition``): each rank forms its block's images and the pairs
within it, and the pair across a block's end needs one image from the next
rank (``exchange_boundary``, one point-to-point transfer per boundary).
"""
from __future__ import annotations

from typing import List, Sequence


def lpt_partition(weights: Sequence[float], nranks: int) -> List[List[int]]:
    """Burst indices per rank by the LPT rule: bursts in decreasing weight
    (ties: lower index first), each to the rank with the least assigned
    weight so far (ties: lower rank).  Each rank's list is in burst order.
    Deterministic, so every rank computes the same partition."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * nranks
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(weights[i])
    return [sorted(p) for p in parts]


def owners(parts: Sequence[Sequence[int]], n: int) -> List[int]:
    """Rank that computes each of the n bursts."""
    own = [-1] * n
    for r, p in enumerate(parts):
        for i in p:
            own[i] = r
    if min(own, default=0) < 0:
        raise ValueError("a burst has no rank")
    return own


def block_partition(n: int, nranks: int) -> List[List[int]]:
    """Indices 0..n-1 in contiguous blocks, one per rank and in order (a
    repeat-pass stack's date order), sizes differing by at most one (the first
    n % nranks blocks one longer)."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    q, r = divmod(n, nranks)
    out, a = [], 0
    for k in range(nranks):
        b = a + q + (1 if k < r else 0)
        out.append(list(range(a, b)))
        a = b
    return out


def exchange_boundary(first_image, recv_buf, rank: int, world: int, dist, group=None):
    """The one transfer a stack dealt in contiguous blocks needs for its
    sequential pairs (k, k+1): every rank but the first sends its first image
    to the previous rank, and every rank but the last receives the next rank's
    first image into `recv_buf`, the second image of the pair across the end
    of its block.  Every rank of a group of two or more takes part.  Returns
    `recv_buf` on the ranks that receive, else None."""
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, first_image, rank - 1, group=group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.irecv, recv_buf, rank + 1, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    return recv_buf if rank < world - 1 else None


def gather_outputs(outs, owner: Sequence[int], rank: int, dist, dst: int = 0, group=None) -> None:
    """Point-to-point gather of burst images to rank `dst`: the owner of
    burst i sends outs[i] (a contiguous tensor) and `dst` receives it into
    its own outs[i] (same shape and dtype).  Every burst computed on `dst`
    stays where it is.  Blocks (the current stream, for NCCL) until this
    rank's transfers are complete."""
    ops = []
    for i, o in enumerate(owner):
        if o == dst:
            continue
        if rank == o:
            ops.append(dist.P2POp(dist.isend, outs[i], dst, group=group))
        elif rank == dst:
            ops.append(dist.P2POp(dist.irecv, outs[i], o, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def ordered_merge(raster, bursts, stream=None) -> None:
    """Merge burst images (DeviceBurst, in global burst order) into the scene
    raster with the reference's rule, on the GPU (srg_merge_device, one launch
    per burst on one stream, so later bursts replace earlier ones)."""
    from . import api
    for db in bursts:
        ncols = db.out.shape[1]
        view = raster[db.firstline:db.firstline + db.nlines, db.out_pix0:db.out_pix0 + ncols]
        api.merge(view, db.out, stream=stream)


class PartitionedScene:
    """One scene's bursts dealt over the ranks of a process group: this
    rank's scene plan over its own bursts (one persistent backprojection
    launch, no raster), the gather of every burst image to rank `dst`, and
    there the ordered merge into `raster`.  Every rank holds the descriptors
    and image buffers of all bursts (``bursts``: DeviceBurst in scene order;
    only its own need range lines); `weights` estimate each burst's work
    (e.g. its executed-term count) and must be the same on every rank.
    Exposes the ``api.Scene`` methods a caller drives a pass with."""

    def __init__(self, bursts, raster, rank: int, world: int, dist, weights, form: int,
                 dst: int = 0, group=None):
        from . import api
        self.bursts, self.raster = list(bursts), raster
        self.rank, self.world, self.dist, self.dst, self.group = rank, world, dist, dst, group
        self.parts = lpt_partition(weights, world)
        self.owner = owners(self.parts, len(self.bursts))
        self.mine = [self.bursts[i] for i in self.parts[rank]]
        self.weights = [float(w) for w in weights]
        self.plan = api.Scene(self.mine, raster=None, form=form) if self.mine else None

    def own_weight(self) -> float:
        return sum(self.weights[i] for i in self.parts[self.rank])

    def run(self, stream=None) -> None:
        """One pass: own bursts, gather to `dst`, ordered merge there, all
        ordered on `stream` (the transfers wait for the backprojection, the
        merge for the transfers)."""
        import torch

        from . import api
        sp = api._stream_ptr(stream)
        if self.plan is not None:
            self.plan.run(sp)
        with torch.cuda.stream(torch.cuda.ExternalStream(sp)):
            gather_outputs([db.out for db in self.bursts], self.owner, self.rank, self.dist,
                           self.dst, self.group)
        if self.rank == self.dst and self.raster is not None:
            ordered_merge(self.raster, self.bursts, stream=sp)

    def run_stages(self, stages: int, stream=None) -> None:
        if self.plan is not None:
            self.plan.run_stages(stages, stream)

    def sync(self, stream=None) -> None:
        import torch
        if self.plan is not None:
            self.plan.sync(stream)
        torch.cuda.synchronize()

    def tune(self, iters: int = 3):
        return self.plan.tune(iters) if self.plan is not None else (-1, 0.0)

    def set_form(self, form: int, tile_cfg: int = -1) -> None:
        if self.plan is not None:
            self.plan.set_form(form, tile_cfg)

    def shape(self) -> int:
        return self.plan.shape() if self.plan is not None else -1

    def tile_shears(self) -> list:
        return self.plan.tile_shears() if self.plan is not None else []
