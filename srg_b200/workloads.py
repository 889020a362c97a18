"""Device-resident synthetic workloads with the shapes of the benchmark
configurations (see scene.py for the geometry and the reference's
derivations of every burst argument).

The range-compressed samples are made on the GPU by forward projection
(``api.forward_project``): each grid pixel of the burst window is a circular
complex Gaussian scatterer (unit power) and a set of point targets carries
+30 dB; the echo of every pixel, weighted by a sinc^2 azimuth antenna pattern
of a 10 m antenna, is added to the two range bins around its slant range in
every pulse.  Atomic accumulation makes the samples reproducible only to
rounding; every comparison in this project is made between outputs computed
from the same device buffer.
"""
from __future__ import annotations

import dataclasses
import time
from typing import List

import numpy as np

from . import api, scene


@dataclasses.dataclass
class Workload:
    name: str
    bursts: List[api.DeviceBurst]
    coefs: list              # torch float64 [nlines][3] per burst (device azimuth centres)
    terms: int               # exact executed-term count of all bursts
    setup_s: float
    description: str

    def descs_bytes(self):
        """Bytes a host-resident copy of the step inputs/outputs moves."""
        h2d = sum(db.burst.numel() * 8 + db.satloc.numel() * 8 + db.dem.numel() * 2
                  for db in self.bursts)
        d2h = sum(db.out.numel() * 8 for db in self.bursts)
        return h2d, d2h


def _reflectivity(torch, shape, seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    s = 1.0 / np.sqrt(2.0)
    re = torch.randn(shape, generator=g, device=device) * s
    im = torch.randn(shape, generator=g, device=device) * s
    return torch.complex(re, im)


def forward_burst(db: api.DeviceBurst, seed: int, ntargets: int = 200, target_db: float = 30.0):
    """Fill db.burst with the forward-projected echo of the synthetic scene."""
    import torch
    b = db.b
    dev = db.out.device
    refl = torch.zeros((b.demlength, b.demwidth), dtype=torch.complex64, device=dev)
    rows = slice(db.firstline, db.firstline + db.nlines)
    refl[rows] = _reflectivity(torch, (db.nlines, b.demwidth), seed, dev)
    rng = np.random.default_rng(seed)
    amp = 10.0 ** (target_db / 20.0)
    lines = rng.integers(db.firstline, db.firstline + db.nlines, ntargets)
    pix = rng.integers(max(db.firstpix, 0), min(db.lastpix, b.demwidth - 1) + 1, ntargets)
    refl[torch.from_numpy(lines).to(dev), torch.from_numpy(pix).to(dev)] = amp
    db.burst.zero_()
    satvel = torch.from_numpy(np.ascontiguousarray(b.satvel)).to(dev)
    # the kernel indexes the reflectivity with grid rows offset by firstline
    api.forward_project(db, refl[rows], satvel)
    torch.cuda.synchronize(dev)


def config1(device="cuda", seed: int = 1001, forward: bool = True) -> Workload:
    """One IW1-sized burst: 1,500 pulses x 21,000 bins -> 2,400 x 1,200 grid at
    0.0001 deg over a volcano DEM (0-2,500 m cone + fBm, Hurst 0.8, 30 m RMS)."""
    import torch
    t0 = time.time()
    b = scene.config1_geometry(seed=seed)
    bt = torch.zeros((b.rawdatalines, b.samples), dtype=torch.complex64, device=device)
    db = api.to_device(b, device=device, burst_tensor=bt)
    if forward:
        forward_burst(db, seed)
    coef = api.line_centres(db)
    terms = api.count_terms([db])
    return Workload("c1", [db], [coef], terms, time.time() - t0,
                    "IW1 burst 1500x21000 complex64 -> 2400x1200 grid at 1e-4 deg, volcano DEM, "
                    "forward-projected scatterers + 200 targets at +30 dB")
