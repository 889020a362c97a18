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
    raster: object = None    # scene raster (device) the bursts merge into, if any
    grid: object = None      # scene.SceneGrid of a multi-burst scene
    extra: dict = dataclasses.field(default_factory=dict)  # workload-specific arrays

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


def _add_targets(db: api.DeviceBurst, refl_buf, rng, ntargets: int, amp: float):
    """Forward-project `ntargets` point targets at random pixels of the burst
    window into db.burst (accumulates)."""
    import torch
    b = db.b
    dev = db.out.device
    refl = refl_buf[:db.nlines]
    refl.zero_()
    lines = rng.integers(0, db.nlines, ntargets)
    pix = rng.integers(max(db.firstpix, 0), min(db.lastpix, b.demwidth - 1) + 1, ntargets)
    refl[torch.from_numpy(lines).to(dev), torch.from_numpy(pix).to(dev)] = amp
    satvel = torch.from_numpy(np.ascontiguousarray(b.satvel)).to(dev)
    api.forward_project(db, refl, satvel)


def config3(device="cuda", seed: int = 1003, ntargets: int = 200, target_db: float = 30.0,
            form=None) -> Workload:
    """A full IW scene: 3 subswaths x 9 bursts of uneven size (P uniform in
    1,380-1,620; S = 18,000 / 21,500 / 25,600), each mapped to its own
    overlapping sub-grid (2,000-2,600 x 1,000-1,300 at 1e-4 deg) of a shared
    volcano DEM, merged in burst order into one scene raster.  Range lines:
    circular complex Gaussian clutter (unit power per sample) plus
    forward-projected point targets at +30 dB."""
    import torch
    from . import _lib
    t0 = time.time()
    grid, bursts = scene.iw_scene(seed=seed, device=device)
    dem_dev = grid.dem
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    maxl = 0
    dbs = []
    for b in bursts:
        P, S = b.rawdatalines, b.samples
        bt = torch.complex(torch.randn((P, S), generator=gen, device=device),
                           torch.randn((P, S), generator=gen, device=device)) * (1.0 / np.sqrt(2.0))
        db = api.to_device(b, device=device, burst_tensor=bt, dem_tensor=dem_dev, narrow_out=True)
        maxl = max(maxl, db.nlines)
        dbs.append(db)
    refl = torch.zeros((maxl, grid.width), dtype=torch.complex64, device=device)
    amp = 10.0 ** (target_db / 20.0)
    for db in dbs:
        _add_targets(db, refl, rng, ntargets, amp)
    del refl
    raster = torch.zeros((grid.length, grid.width), dtype=torch.complex64, device=device)
    torch.cuda.synchronize(device)
    sc = api.Scene(dbs, raster=raster, form=_lib.FORM_SPLIT if form is None else form)
    terms = sc.terms()
    wl = Workload("c3", dbs, [], terms, time.time() - t0,
                  "IW scene: 3 subswaths x 9 bursts (P 1380-1620, S 18000/21500/25600 complex64, "
                  f"{sum(db.burst.numel() * 8 for db in dbs) / 1e9:.2f} GB), sub-grids 2000-2600 x "
                  f"1000-1300 at 1e-4 deg on a shared {grid.width}x{grid.length} volcano DEM, "
                  "merged in burst order", raster=raster, grid=grid)
    wl.plan = sc
    # host copy of the shared DEM for the file-based entry
    host_dem = dem_dev.cpu().numpy()
    for b in bursts:
        b.dem = host_dem
    return wl


def iw_bursts(indices=(0, 1, 2), device="cuda", seed: int = 1003, ntargets: int = 200,
              target_db: float = 30.0):
    """Selected bursts of the IW scene (configuration 3) on their own, for
    checks at full size: the scene's geometry and shared volcano DEM, each
    burst's range lines circular complex Gaussian clutter plus `ntargets`
    forward-projected point targets at +30 dB (the scene's statistics; the
    samples are drawn per burst, so they are not the ones config3 draws).
    Indices 0, 1, 2 are the first burst of subswaths 1, 2, 3.  Returns
    (SceneGrid with a host DEM, [DeviceBurst]); each burst's `b.dem` is the
    host DEM and `b.burst` is left empty (the samples live on the device)."""
    import torch
    grid, bursts = scene.iw_scene(seed=seed, device=device)
    dem_dev = grid.dem
    host_dem = dem_dev.cpu().numpy()
    amp = 10.0 ** (target_db / 20.0)
    dbs = []
    for i in indices:
        b = bursts[i]
        b.dem = host_dem
        gen = torch.Generator(device=device)
        gen.manual_seed(seed * 100 + i)
        P, S = b.rawdatalines, b.samples
        bt = torch.complex(torch.randn((P, S), generator=gen, device=device),
                           torch.randn((P, S), generator=gen, device=device)) * (1.0 / np.sqrt(2.0))
        db = api.to_device(b, device=device, burst_tensor=bt, dem_tensor=dem_dev, narrow_out=True)
        refl = torch.zeros((db.nlines, grid.width), dtype=torch.complex64, device=device)
        _add_targets(db, refl, np.random.default_rng(seed * 100 + i), ntargets, amp)
        dbs.append(db)
    torch.cuda.synchronize(device)
    grid.dem = host_dem
    return grid, dbs


def config4(device="cuda", seed: int = 1004, acquisitions: int = 32, bperp_max: float = 150.0,
            along_max: float = 5.0, los_max: float = 0.10, depth: float = 3000.0,
            ntargets: int = 200, target_db: float = 30.0, form=None) -> Workload:
    """Repeat-pass stack: `acquisitions` passes over the config-1 footprint
    (1,500 pulses x 21,000 bins each, common 2,400 x 1,200 grid at 1e-4 deg
    over the volcano DEM).  Pass k has its state vectors displaced by a
    perpendicular baseline drawn from U[-bperp_max, bperp_max] m and its pulse
    times shifted by an along-track offset from U[-along_max, along_max] m;
    the scene (one circular Gaussian scatterer per grid pixel plus point
    targets at +30 dB, identical in every pass) has moved by k/(n-1) of a Mogi
    source's range change (depth 3 km below the summit, max 10 cm of line of
    sight).  All passes form one scene plan without a raster: one batched
    backprojection launch writes every pass's image on the common grid."""
    import torch
    from . import _lib
    t0 = time.time()
    base = scene.config1_geometry(seed=seed)
    rng = np.random.default_rng(seed)
    e_perp, speed = scene.baseline_frame(base)
    bperp = rng.uniform(-bperp_max, bperp_max, acquisitions)
    along = rng.uniform(-along_max, along_max, acquisitions)
    bperp[0] = along[0] = 0.0  # the first pass is the reference orbit
    drange = scene.mogi_range_change(base, depth=depth, los_max=los_max)
    L, W = base.demlength, base.demwidth
    dem_t = torch.from_numpy(np.ascontiguousarray(base.dem)).to(device)
    refl = _reflectivity(torch, (L, W), seed, device)
    amp = 10.0 ** (target_db / 20.0)
    lines = rng.integers(0, L, ntargets)
    pix = rng.integers(0, W, ntargets)
    refl[torch.from_numpy(lines).to(device), torch.from_numpy(pix).to(device)] = amp
    dr_t = torch.from_numpy(drange).to(device)
    dbs = []
    for k in range(acquisitions):
        b = scene.make_geometry(pulses=base.rawdatalines, samples=base.samples, width=W, length=L,
                                spacing=abs(base.deltalat), centre_height=1000.0,
                                grid_centre=scene.grid_centre(base),
                                position_offset=bperp[k] * e_perp, along_offset=along[k] / speed)
        # the common grid, to the bit
        b.firstlat, b.firstlon, b.latlons = base.firstlat, base.firstlon, base.latlons.copy()
        b.dem = base.dem
        bt = torch.zeros((b.rawdatalines, b.samples), dtype=torch.complex64, device=device)
        db = api.to_device(b, device=device, burst_tensor=bt, dem_tensor=dem_t)
        rows = slice(db.firstline, db.firstline + db.nlines)
        offs = (dr_t[rows] * (k / max(1, acquisitions - 1))).contiguous()
        satvel = torch.from_numpy(np.ascontiguousarray(b.satvel)).to(device)
        api.forward_project(db, refl[rows], satvel, range_offset=offs)
        dbs.append(db)
    torch.cuda.synchronize(device)
    sc = api.Scene(dbs, raster=None, form=_lib.FORM_SPLIT if form is None else form)
    terms = sc.terms()
    wl = Workload("c4", dbs, [], terms, time.time() - t0,
                  f"repeat-pass stack: {acquisitions} passes of 1500 x 21000 complex64 "
                  f"({sum(db.burst.numel() * 8 for db in dbs) / 1e9:.2f} GB) onto a common "
                  f"{W}x{L} grid at 1e-4 deg, perpendicular baselines U[+-{bperp_max:g} m], "
                  f"along-track U[+-{along_max:g} m], Mogi source {depth / 1000:g} km deep, "
                  f"{los_max * 100:g} cm max LOS growing linearly; then crossmul of "
                  f"{acquisitions - 1} sequential pairs")
    wl.plan = sc
    wl.extra = {"range_change": drange, "bperp": bperp, "along": along,
                "wvl": base.wvl, "acquisitions": acquisitions}
    return wl
