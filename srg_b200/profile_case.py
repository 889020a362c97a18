"""Profiling driver: a fixed workload and a list of kernel shapes, one
warm-up launch then one measured launch per shape, nothing else on the GPU.

  python -m srg_b200.profile_case [--samples random|forward] SHAPE [SHAPE ...]

SHAPE indexes srg_b200._lib.tile_configs().  Under ncu, skip the warm-ups with
`-s <number of shapes + 4>` (count includes the azimuth-centre and term-count
launches of the set-up) or select by kernel name.
"""
from __future__ import annotations

import argparse

from . import _lib, api, scene, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("shapes", type=int, nargs="*")
    ap.add_argument("--samples", default="random", choices=["random", "forward"])
    ap.add_argument("--seed", type=int, default=1001)
    a = ap.parse_args()
    import torch
    if a.samples == "forward":
        wl = workloads.config1(seed=a.seed)
        db, coef = wl.bursts[0], wl.coefs[0]
    else:
        b = scene.config1_geometry(seed=a.seed)
        g = torch.Generator(device="cuda")
        g.manual_seed(a.seed)
        bt = torch.complex(torch.randn(b.rawdatalines, b.samples, device="cuda", generator=g),
                           torch.randn(b.rawdatalines, b.samples, device="cuda", generator=g))
        db = api.to_device(b, burst_tensor=bt)
        coef = api.line_centres(db)
    cfgs = _lib.tile_configs()
    shapes = a.shapes or [0]
    for s in shapes:
        api.backproject([db], form=cfgs[s][1], tile_cfg=s, coefs=[coef])
    for s in shapes:
        api.backproject([db], form=cfgs[s][1], tile_cfg=s, coefs=[coef])
    torch.cuda.synchronize()
    print("ok", shapes)


if __name__ == "__main__":
    main()
