"""Profiling driver: a fixed workload and a list of kernel shapes, one
warm-up launch then one measured launch per shape, nothing else on the GPU.

  python -m srg_b200.profile_case [--workload c1|c3] [--samples random|forward] SHAPE [SHAPE ...]

SHAPE indexes srg_b200._lib.tile_configs().  c1: one IW1-sized burst; c3: the
27-burst IW scene, backprojection stage of its scene plan only.  Under ncu,
select the backprojection kernels by name (regex:bp_) and skip the warm-up
launches with -s <number of shapes>.
"""
from __future__ import annotations

import argparse

from . import _lib, api, scene, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("shapes", type=int, nargs="*")
    ap.add_argument("--samples", default="random", choices=["random", "forward"])
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--workload", default="c1", choices=["c1", "c3"])
    a = ap.parse_args()
    import torch
    cfgs = _lib.tile_configs()
    shapes = a.shapes or [0]
    if a.workload == "c3":
        wl = workloads.config3(seed=1003 if a.seed is None else a.seed)
        plan = wl.plan
        for rep in range(2):  # warm-up, then measured
            for s in shapes:
                plan.set_form(cfgs[s][1], s)
                plan.run_stages(1 | 2, 0)
        plan.sync(0)
        print("ok", shapes)
        return
    if a.seed is None:
        a.seed = 1001
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
    for s in shapes:
        api.backproject([db], form=cfgs[s][1], tile_cfg=s, coefs=[coef])
    for s in shapes:
        api.backproject([db], form=cfgs[s][1], tile_cfg=s, coefs=[coef])
    torch.cuda.synchronize()
    print("ok", shapes)


if __name__ == "__main__":
    main()
