"""Synthetic Sentinel-1-like bursts for the backprojection path.

Builds, deterministically from a seed, every argument of the per-burst
entry ``azimuth_compress_`` (sentinel/azimuth_compress.cu:181-214) the way the
reference's drivers derive them:

* orbit state vectors every 10 s around the burst (11 of them, as
  sentinel/getburststatevectors.f90:112-128 writes), from a circular orbit of
  radius 7,071 km and inclination 98.18 deg, expressed in the rotating (ECEF)
  frame;
* per-pulse satellite positions/velocities by 4-point Hermite interpolation of
  those vectors, with the window rule of sentinel/sentineltimingsub.f90:55-66
  and the text quantisation of its write (f16.7 m, f14.8 m/s);
* burst-centre position/velocity with the clamped window of
  sentinel/intp_orbit.f90;
* rngstart/rngend/dmrg/tmid as sentinel/backprojectcpusub.f90:216-227 and the
  aperture length as backprojectcpusub.f90:195-211;
* an int16 ellipsoid-height DEM (flat, or a volcano cone plus fBm roughness)
  on a lat/lon grid whose centre is the beam centre of the burst.

Range-compressed samples are synthesised here for point targets (numpy); the
distributed-scatterer forward projection of the large configurations runs on
the GPU (``srg_b200.api.forward_project``).

Everything is float64 numpy; no value here feeds a parity claim except
through arrays that are handed, bit for bit, to both the CUDA path and the
oracle.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

C_LIGHT = 299792458.0
WGS84_A = 6378137.0
WGS84_E2 = 0.0066943799901499996
GM_EARTH = 3.986004418e14
OMEGA_EARTH = 7.2921159e-5

# Radar constants of the synthetic configurations.
WAVELENGTH = 0.0554658
PRF = 1717.13
RANGE_FS = 64.345e6
NEAR_RANGE = 800.0e3
ORBIT_RADIUS = 7071.0e3
ORBIT_INCL_DEG = 98.18
SV_SPACING = 10.0


@dataclasses.dataclass
class Burst:
    """All arguments of one ``azimuth_compress_`` call (names as the reference)."""

    burst: np.ndarray            # [P][S] complex64 range-compressed lines
    satloc: np.ndarray           # [P][3] float64 ECEF position per pulse
    satvel: np.ndarray           # [P][3] float64 ECEF velocity per pulse
    pulse_time: np.ndarray       # [P] float64 line times (s)
    demwidth: int
    demlength: int
    deltalat: float              # deg (negative: lines run north to south)
    deltalon: float
    firstlat: float
    firstlon: float
    latlons: np.ndarray          # [4] min lat, max lat, min lon, max lon
    timeorbit: np.ndarray        # [n]
    xx: np.ndarray               # [n][3]
    vv: np.ndarray               # [n][3]
    rngstart: float
    rngend: float
    tstart: float
    tend: float
    tmid: float
    xyz_mid: np.ndarray          # [3]
    vel_mid: np.ndarray          # [3]
    dtaz: float
    dmrg: float
    wvl: float
    aperture: int
    iaperture: int
    angc0: float
    angc1: float
    prf: float
    dem: Optional[np.ndarray] = None     # [demlength][demwidth] int16 (full DEM)
    targets: Optional[np.ndarray] = None  # [T][3] (line, pixel, amplitude) of point targets
    pulses: int = 0   # pulse count when the samples live only on the device (burst has 0 rows)

    @property
    def rawdatalines(self) -> int:
        return int(self.pulses or self.burst.shape[0])

    @property
    def samples(self) -> int:
        return int(self.burst.shape[1])

    @property
    def numstatevec(self) -> int:
        return int(self.timeorbit.shape[0])


# --------------------------------------------------------------------------
# orbit


@dataclasses.dataclass
class CircularOrbit:
    radius: float = ORBIT_RADIUS
    incl_deg: float = ORBIT_INCL_DEG
    raan: float = 0.0
    u0: float = 0.0          # argument of latitude at epoch
    epoch: float = 0.0       # s; Earth rotation angle is zero here
    ascending: bool = True

    @property
    def mean_motion(self) -> float:
        return math.sqrt(GM_EARTH / self.radius ** 3)

    def state(self, t):
        """ECEF position and velocity at times t (array) -> ([N,3], [N,3])."""
        t = np.asarray(t, dtype=np.float64)
        n = self.mean_motion
        u = self.u0 + n * (t - self.epoch)
        inc = math.radians(self.incl_deg)
        co, so = math.cos(self.raan), math.sin(self.raan)
        ci, si = math.cos(inc), math.sin(inc)
        cu, su = np.cos(u), np.sin(u)
        r = self.radius
        xi = np.stack([r * (co * cu - so * su * ci), r * (so * cu + co * su * ci), r * su * si], -1)
        vi = np.stack([r * n * (-co * su - so * cu * ci), r * n * (-so * su + co * cu * ci),
                       r * n * cu * si], -1)
        th = OMEGA_EARTH * (t - self.epoch)
        ct, st = np.cos(th), np.sin(th)
        # rotate inertial -> ECEF by -theta about z
        x = np.stack([ct * xi[..., 0] + st * xi[..., 1], -st * xi[..., 0] + ct * xi[..., 1],
                      xi[..., 2]], -1)
        vrot = np.stack([ct * vi[..., 0] + st * vi[..., 1], -st * vi[..., 0] + ct * vi[..., 1],
                         vi[..., 2]], -1)
        # v_ecef = R v_i - omega x x_ecef
        v = vrot + np.stack([OMEGA_EARTH * x[..., 1], -OMEGA_EARTH * x[..., 0],
                             np.zeros_like(x[..., 2])], -1)
        return x, v


def hermite4(ts, xs, vs, t):
    """4-point position/velocity Hermite interpolation.

    Same basis as sentinel/orbithermite.f:21-70 (value f0/f1 and derivative
    g0/g1 weights built on the Lagrange polynomials h and their derivatives).
    ts: [..., 4]; xs, vs: [..., 4, 3]; t: [...].  Returns ([..., 3], [..., 3]).
    """
    ts = np.asarray(ts, np.float64)
    t = np.asarray(t, np.float64)[..., None]
    n = 4
    inv = np.zeros(ts.shape[:-1] + (n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                inv[..., i, j] = 1.0 / (ts[..., i] - ts[..., j])
    s = inv.sum(-1)  # sum_j!=i 1/(t_i - t_j)
    dt = t - ts
    f0 = 1.0 - 2.0 * dt * s
    f1 = dt
    h = np.ones_like(ts)
    for i in range(n):
        for k in range(n):
            if k != i:
                h[..., i] = h[..., i] * (t[..., 0] - ts[..., k]) / (ts[..., i] - ts[..., k])
    hd = np.zeros_like(ts)
    for i in range(n):
        acc = np.zeros(ts.shape[:-1])
        for j in range(n):
            if j == i:
                continue
            q = np.ones(ts.shape[:-1])
            for k in range(n):
                if k != i and k != j:
                    q = q * (t[..., 0] - ts[..., k]) / (ts[..., i] - ts[..., k])
            acc = acc + inv[..., i, j] * q
        hd[..., i] = acc
    g1 = h + 2.0 * dt * hd
    g0 = 2.0 * (f0 * hd - h * s)
    xq = np.sum((xs * f0[..., None] + vs * f1[..., None]) * (h * h)[..., None], axis=-2)
    vq = np.sum((xs * g0[..., None] + vs * g1[..., None]) * h[..., None], axis=-2)
    return xq, vq


def interp_pulses(timeorbit, xx, vv, times):
    """Per-pulse orbit: window start int((t - t1)/dt) - 1 (1-based), unclamped,
    as sentinel/sentineltimingsub.f90:61-63."""
    dt = timeorbit[1] - timeorbit[0]
    loc = np.trunc((times - timeorbit[0]) / dt).astype(np.int64)
    s = loc - 2
    if np.any(s < 0) or np.any(s + 3 >= len(timeorbit)):
        raise ValueError("pulse times fall outside the state-vector window")
    idx = s[:, None] + np.arange(4)[None, :]
    return hermite4(timeorbit[idx], xx[idx], vv[idx], times)


def intp_orbit(timeorbit, xx, vv, t):
    """Clamped-window Hermite as sentinel/intp_orbit.f90:1-25."""
    n = len(timeorbit)
    loc = int((t - timeorbit[0]) / (timeorbit[1] - timeorbit[0]))
    loc = min(max(loc, 2), n - 2)
    s = loc - 2
    xq, vq = hermite4(timeorbit[s:s + 4], xx[s:s + 4], vv[s:s + 4], np.float64(t))
    return xq, vq


def quantise_positions(x, v):
    """Round-trip through the text format f16.7 / f14.8
    (sentinel/sentineltimingsub.f90:65, read back at backprojectcpusub.f90:179)."""
    xq = np.array([[float(f"{c:.7f}") for c in row] for row in x])
    vq = np.array([[float(f"{c:.8f}") for c in row] for row in v])
    return xq, vq


# --------------------------------------------------------------------------
# geodesy


def llh_to_ecef(lat_deg, lon_deg, h):
    lat = np.radians(lat_deg)
    lon = np.radians(lon_deg)
    s = np.sin(lat)
    re = WGS84_A / np.sqrt(1.0 - WGS84_E2 * s * s)
    x = (re + h) * np.cos(lat) * np.cos(lon)
    y = (re + h) * np.cos(lat) * np.sin(lon)
    z = (re * (1.0 - WGS84_E2) + h) * s
    return np.stack([x, y, z], -1)


def ecef_to_llh(p):
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    lon = np.arctan2(y, x)
    rho = np.hypot(x, y)
    lat = np.arctan2(z, rho * (1 - WGS84_E2))
    for _ in range(8):
        s = np.sin(lat)
        re = WGS84_A / np.sqrt(1 - WGS84_E2 * s * s)
        h = rho / np.cos(lat) - re
        lat = np.arctan2(z, rho * (1 - WGS84_E2 * re / (re + h)))
    s = np.sin(lat)
    re = WGS84_A / np.sqrt(1 - WGS84_E2 * s * s)
    h = rho / np.cos(lat) - re
    return np.degrees(lat), np.degrees(lon), h


def zero_doppler_point(sat, vel, slant, height, right=True):
    """Ground point at the given slant range and ellipsoid height in the plane
    through `sat` perpendicular to `vel` (zero Doppler), right-looking."""
    vhat = vel / np.linalg.norm(vel)
    down = -sat / np.linalg.norm(sat)
    down = down - np.dot(down, vhat) * vhat
    down /= np.linalg.norm(down)
    side = np.cross(vhat, down)          # right of track for a right-looking SAR
    if not right:
        side = -side
    ang = 0.5
    for _ in range(60):
        p = sat + slant * (math.cos(ang) * down + math.sin(ang) * side)
        _, _, h = ecef_to_llh(p)
        # d h / d ang by finite difference
        p2 = sat + slant * (math.cos(ang + 1e-7) * down + math.sin(ang + 1e-7) * side)
        _, _, h2 = ecef_to_llh(p2)
        dh = (h2 - h) / 1e-7
        step = (h - height) / dh
        ang -= step
        if abs(step) < 1e-13:
            break
    return sat + slant * (math.cos(ang) * down + math.sin(ang) * side)


# --------------------------------------------------------------------------
# DEM


def fbm_surface(rng, ny, nx, hurst, rms):
    """Spectral-synthesis fractional Brownian surface with the given RMS."""
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    ph = rng.standard_normal((ny, kx.shape[1])) + 1j * rng.standard_normal((ny, kx.shape[1]))
    surf = np.fft.irfft2(amp * ph, s=(ny, nx))
    surf -= surf.mean()
    surf *= rms / max(surf.std(), 1e-30)
    return surf


def volcano_dem_torch(seed: int, ny, nx, device, peak=2500.0, base=0.0, radius_frac=0.45,
                      hurst=0.8, rms=30.0):
    """The same surface as volcano_dem, synthesised on a torch device (for
    scene-sized grids); returns an int16 tensor on that device."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    cy, cx = (ny - 1) / 2.0, (nx - 1) / 2.0
    rad = radius_frac * min(ny, nx) * 1.6
    yy = ((torch.arange(ny, device=device, dtype=torch.float32) - cy) / rad)[:, None]
    xx = ((torch.arange(nx, device=device, dtype=torch.float32) - cx) / rad)[None, :]
    h = base + peak * torch.clamp(1.0 - torch.sqrt(yy * yy + xx * xx), 0.0, 1.0)
    ky = torch.fft.fftfreq(ny, device=device)[:, None]
    kx = torch.fft.rfftfreq(nx, device=device)[None, :]
    k = torch.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    ph = torch.complex(torch.randn(amp.shape, generator=g, device=device),
                       torch.randn(amp.shape, generator=g, device=device))
    surf = torch.fft.irfft2(amp * ph, s=(ny, nx))
    surf = surf - surf.mean()
    surf = surf * (rms / torch.clamp(surf.std(), min=1e-30))
    return torch.clamp(torch.round(h + surf), -32768, 32767).to(torch.int16)


def volcano_dem(rng, ny, nx, peak=2500.0, base=0.0, radius_frac=0.45, hurst=0.8, rms=30.0,
                max_fbm_points: int = 4_000_000):
    """Volcano cone (0..peak m) plus fBm roughness (Hurst `hurst`, `rms` m).
    The fBm is synthesised at full resolution up to `max_fbm_points`, beyond
    that on a coarser grid and interpolated bilinearly (its power at the
    finest scales is negligible for H = 0.8)."""
    cy, cx = (ny - 1) / 2.0, (nx - 1) / 2.0
    rad = radius_frac * min(ny, nx) * 1.6
    yy = ((np.arange(ny, dtype=np.float32) - cy) / rad)[:, None]
    xx = ((np.arange(nx, dtype=np.float32) - cx) / rad)[None, :]
    h = base + peak * np.clip(1.0 - np.sqrt(yy * yy + xx * xx), 0.0, 1.0)
    f = 1
    while (ny // f) * (nx // f) > max_fbm_points:
        f *= 2
    if f == 1:
        rough = fbm_surface(rng, ny, nx, hurst, rms)
    else:
        from scipy import ndimage
        coarse = fbm_surface(rng, -(-ny // f), -(-nx // f), hurst, rms).astype(np.float32)
        rough = ndimage.zoom(coarse, f, order=1)[:ny, :nx]
    h = h + rough
    return np.clip(np.rint(h), -32768, 32767).astype(np.int16)


# --------------------------------------------------------------------------
# burst geometry


def aperture_points(satvel, rngstart, wvl, prf, angc1=0.0):
    """sentinel/backprojectcpusub.f90:195-211 (TOPS aperture, 50 % of nominal)."""
    re, ht = 6378137.0, 700000.0
    p = satvel.shape[0]
    v = satvel[p // 2 - 1]  # Fortran satvel(:, rawdatalines/2)
    vmag = math.sqrt(float(np.dot(v, v))) * (re / (re + ht))
    pi = 4.0 * math.atan2(1.0, 1.0)
    aperturetime = (rngstart * wvl / 2 / vmag / vmag * prf) / (1.0 + rngstart * angc1 * pi / 180.0 / vmag)
    return int(aperturetime * prf * 0.5)


def make_geometry(*, pulses: int, samples: int, width: int, length: int, spacing: float,
                  near_range: float = NEAR_RANGE, wvl: float = WAVELENGTH, prf: float = PRF,
                  fs: float = RANGE_FS, lat0: float = 19.4, tmid_nominal: float = 43200.25,
                  centre_height: float = 0.0, aperture: Optional[int] = None,
                  angc0: float = 0.0, angc1: float = 0.0, quantise: bool = True,
                  grid_centre: Optional[tuple] = None, orbit: Optional[CircularOrbit] = None,
                  along_offset: float = 0.0, position_offset=None) -> Burst:
    """Orbit, pulses and grid of one burst; samples are left zero.
    along_offset (s) shifts the pulse times along the orbit; position_offset
    (ECEF metres) displaces every state vector (a repeat-pass baseline)."""
    if orbit is None:
        inc = math.radians(ORBIT_INCL_DEG)
        u0 = math.asin(math.sin(math.radians(lat0)) / math.sin(inc))
        orbit = CircularOrbit(u0=u0, epoch=tmid_nominal)
    dtaz = 1.0 / prf
    tstart = tmid_nominal - 0.5 * (pulses - 1) * dtaz + along_offset
    tend = tstart + (pulses - 1) * dtaz
    tmid = 0.5 * (tstart + tend)
    t0 = math.floor((tstart - 30.0) / SV_SPACING) * SV_SPACING + SV_SPACING
    timeorbit = t0 + SV_SPACING * np.arange(11, dtype=np.float64)
    xx, vv = orbit.state(timeorbit)
    if position_offset is not None:
        xx = xx + np.asarray(position_offset, np.float64)[None, :]
    ptime = tstart + np.arange(pulses, dtype=np.float64) * dtaz
    sx, sv = interp_pulses(timeorbit, xx, vv, ptime)
    if quantise:
        sx, sv = quantise_positions(sx, sv)
    xyz_mid, vel_mid = intp_orbit(timeorbit, xx, vv, tmid)
    dmrg = C_LIGHT / 2.0 / fs
    rngstart = near_range
    rngend = rngstart + (samples - 1) * dmrg
    if grid_centre is None:
        smid, vmid = orbit.state(np.array([tmid_nominal]))
        pc = zero_doppler_point(smid[0], vmid[0], 0.5 * (rngstart + rngend), centre_height)
        clat, clon, _ = ecef_to_llh(pc)
        clat, clon = float(clat), float(clon)
    else:
        clat, clon = grid_centre
    deltalat = -spacing
    deltalon = spacing
    firstlat = clat + 0.5 * (length - 1) * spacing
    firstlon = clon - 0.5 * (width - 1) * spacing
    # lat/lon box covering the whole grid (firstpix = 0, lastpix clamps to W)
    latlons = np.array([firstlat + (length - 0.5) * deltalat, firstlat + 0.25 * spacing,
                        firstlon + 0.25 * spacing, firstlon + (width + 0.5) * deltalon])
    if aperture is None:
        aperture = aperture_points(sv, rngstart, wvl, prf, angc1)
    return Burst(
        burst=np.zeros((pulses, samples), np.complex64), satloc=np.ascontiguousarray(sx),
        satvel=np.ascontiguousarray(sv), pulse_time=ptime, demwidth=width, demlength=length,
        deltalat=deltalat, deltalon=deltalon, firstlat=firstlat, firstlon=firstlon,
        latlons=latlons, timeorbit=timeorbit, xx=np.ascontiguousarray(xx),
        vv=np.ascontiguousarray(vv), rngstart=rngstart, rngend=rngend, tstart=tstart, tend=tend,
        tmid=tmid, xyz_mid=np.ascontiguousarray(xyz_mid), vel_mid=np.ascontiguousarray(vel_mid),
        dtaz=dtaz, dmrg=dmrg, wvl=wvl, aperture=int(aperture), iaperture=0, angc0=angc0,
        angc1=angc1, prf=prf)


def grid_ecef(b: Burst, lines, pixels, heights):
    lat = b.firstlat + np.asarray(lines, np.float64) * b.deltalat
    lon = b.firstlon + np.asarray(pixels, np.float64) * b.deltalon
    return llh_to_ecef(lat, lon, np.asarray(heights, np.float64))


def grid_centre(b: Burst):
    """(lat, lon) of the grid's centre pixel."""
    return (b.firstlat + 0.5 * (b.demlength - 1) * b.deltalat,
            b.firstlon + 0.5 * (b.demwidth - 1) * b.deltalon)


def baseline_frame(b: Burst):
    """Unit vector normal to both the line of sight to the grid centre and
    the velocity at mid-burst (the direction of a perpendicular baseline),
    and the orbital speed (m/s)."""
    clat, clon = grid_centre(b)
    h = float(b.dem[b.demlength // 2, b.demwidth // 2]) if b.dem is not None else 0.0
    p = llh_to_ecef(clat, clon, h)
    los = p - b.xyz_mid
    los /= np.linalg.norm(los)
    v = np.asarray(b.vel_mid, np.float64)
    e = np.cross(los, v / np.linalg.norm(v))
    return e / np.linalg.norm(e), float(np.linalg.norm(v))


def mogi_range_change(b: Burst, depth: float = 3000.0, los_max: float = 0.10) -> np.ndarray:
    """Range change (m, float32 [demlength][demwidth]) of every grid pixel due
    to a Mogi point source `depth` metres below the ellipsoid under the grid
    centre: surface displacement u = C (x - s) / |x - s|^3 (the point-source
    field of an elastic half-space, Mogi 1958), projected on the unit vector
    from the pixel to the mid-burst satellite position, negated (uplift toward
    the radar shortens the range), scaled so that max |change| = los_max."""
    L, W = b.demlength, b.demwidth
    clat, clon = grid_centre(b)
    src = llh_to_ecef(clat, clon, -depth)
    lat = b.firstlat + np.arange(L, dtype=np.float64)[:, None] * b.deltalat
    lon = b.firstlon + np.arange(W, dtype=np.float64)[None, :] * b.deltalon
    P = llh_to_ecef(np.broadcast_to(lat, (L, W)), np.broadcast_to(lon, (L, W)),
                    b.dem.astype(np.float64))
    d = P - src
    u = d / (np.linalg.norm(d, axis=-1, keepdims=True) ** 3)
    s = np.asarray(b.xyz_mid, np.float64) - P
    s /= np.linalg.norm(s, axis=-1, keepdims=True)
    dr = -(u * s).sum(-1)
    return (dr * (los_max / np.abs(dr).max())).astype(np.float32)


# --------------------------------------------------------------------------
# samples


def _sinc(x):
    return np.sinc(x)


def add_point_targets(b: Burst, positions, amplitudes, taps: int = 16, antenna: float = 10.0):
    """Forward-project point targets into the range-compressed lines.

    Per pulse each target adds sinc(bin - r) * exp(-j 4 pi R / lambda), weighted
    by a sinc^2 azimuth antenna pattern of a `antenna`-metre aperture, with a
    Hann-tapered +-`taps` bin range response.
    """
    P, S = b.burst.shape
    out = b.burst
    offs = np.arange(-taps, taps + 1)
    for pos, amp in zip(np.asarray(positions), np.asarray(amplitudes)):
        d = pos[None, :] - b.satloc
        R = np.sqrt(np.sum(d * d, axis=1))
        vhat = b.satvel / np.linalg.norm(b.satvel, axis=1)[:, None]
        sin_sq = np.sum(d * vhat, axis=1) / R
        w_az = _sinc(antenna * sin_sq / b.wvl) ** 2
        r = (R - b.rngstart) / b.dmrg
        base = np.floor(r).astype(np.int64)
        bins = base[:, None] + offs[None, :]
        x = bins - r[:, None]
        win = 0.5 * (1.0 + np.cos(np.pi * np.clip(x / (taps + 1), -1, 1)))
        val = _sinc(x) * win * w_az[:, None]
        ph = np.exp(-1j * (4.0 * np.pi / b.wvl) * R)
        contrib = (amp * val * ph[:, None]).astype(np.complex64)
        ok = (bins >= 0) & (bins < S)
        rows = np.broadcast_to(np.arange(P)[:, None], bins.shape)
        np.add.at(out, (rows[ok], bins[ok]), contrib[ok])


def add_noise(b: Burst, rng, snr_db: float, ref_amplitude: float = 1.0):
    """Complex Gaussian noise; SNR is the per-sample ratio of a unit target's
    peak power (ref_amplitude^2) to the noise power."""
    sigma2 = ref_amplitude ** 2 / 10 ** (snr_db / 10.0)
    s = math.sqrt(sigma2 / 2.0)
    n = rng.standard_normal(b.burst.shape + (2,), dtype=np.float32) * np.float32(s)
    b.burst += n[..., 0] + 1j * n[..., 1]


# --------------------------------------------------------------------------
# configurations


def config0_point_targets(seed: int = 1000, pulses: int = 1024, samples: int = 4096,
                          width: int = 256, length: int = 256, spacing: float = 0.0002,
                          ntargets: int = 64, height: float = 500.0, snr_db: float = 10.0,
                          quantise: bool = True) -> Burst:
    """64 point targets on flat 500 m terrain, 10 dB SNR (configuration 0).
    Targets sit on pixel centres whose aperture centre is well inside the
    burst, so that every one of them is formed."""
    rng = np.random.default_rng(seed)
    b = make_geometry(pulses=pulses, samples=samples, width=width, length=length,
                      spacing=spacing, centre_height=height, quantise=quantise)
    b.dem = np.full((length, width), int(height), np.int16)
    ok = formed_mask_estimate(b, margin=24)
    ok[:, :8] = False
    ok[:, -8:] = False
    ok[:8] = False
    ok[-8:] = False
    cand = np.argwhere(ok)
    order = rng.permutation(len(cand))
    chosen = []
    for i in order:  # keep targets at least 6 pixels apart so each peak is its own
        y, x = cand[i]
        if all(max(abs(y - cy), abs(x - cx)) >= 6 for cy, cx in chosen):
            chosen.append((y, x))
            if len(chosen) == ntargets:
                break
    pick = np.array(chosen)
    lines, pixels = pick[:, 0], pick[:, 1]
    amps = np.ones(ntargets)
    pos = grid_ecef(b, lines, pixels, np.full(ntargets, height))
    add_point_targets(b, pos, amps)
    add_noise(b, rng, snr_db)
    b.targets = np.stack([lines, pixels, amps], -1)
    return b


def formed_mask_estimate(b: Burst, margin: int = 0):
    """Pixels whose nearest-approach pulse lies inside
    (aperture/2 + margin, P - aperture/2 - margin): an estimate of the formed
    region used to place synthetic targets (the exact one is the backprojector's)."""
    P = b.rawdatalines
    h = 0.0 if b.dem is None else b.dem.astype(np.float64)
    ll, pp = np.mgrid[0:b.demlength, 0:b.demwidth]
    pts = grid_ecef(b, ll, pp, np.broadcast_to(h, ll.shape)).reshape(-1, 3)
    sub = b.satloc[::4]
    vel = b.satvel[::4]
    best = np.empty(len(pts), np.int64)
    for i0 in range(0, len(pts), 8192):
        d = pts[i0:i0 + 8192, None, :] - sub[None]
        dop = np.abs(np.sum(d * vel[None], axis=-1))
        best[i0:i0 + 8192] = np.argmin(dop, axis=1) * 4
    lo, hi = b.aperture // 2 + margin, P - b.aperture // 2 - margin
    return ((best > lo) & (best < hi)).reshape(b.demlength, b.demwidth)


def formed_line_band(b: Burst):
    """Approximate range of grid lines whose aperture centre lies inside
    (aperture/2, P - aperture/2), from the zero-Doppler time of the grid centre
    column.  Used only to place synthetic targets."""
    P = b.rawdatalines
    lines = np.arange(b.demlength)
    pix = np.full_like(lines, b.demwidth // 2)
    h = 0.0 if b.dem is None else float(np.median(b.dem))
    pts = grid_ecef(b, lines, pix, np.full(lines.shape, h))
    # zero-Doppler pulse index by nearest approach
    d = pts[:, None, :] - b.satloc[None, ::8, :]
    dop = np.sum(d * b.satvel[None, ::8, :], axis=-1)
    k = np.argmin(np.abs(dop), axis=1) * 8
    ok = (k > b.aperture // 2 + 4) & (k < P - b.aperture // 2 - 4)
    if not np.any(ok):
        return 0, 0
    idx = np.nonzero(ok)[0]
    return int(idx.min()), int(idx.max())


def config1_geometry(seed: int = 1001, pulses: int = 1500, samples: int = 21000,
                     width: int = 2400, length: int = 1200, spacing: float = 0.0001,
                     quantise: bool = True, **kw) -> Burst:
    """IW1-sized burst over a volcano DEM (configuration 1); samples are
    produced on the GPU by forward projection."""
    rng = np.random.default_rng(seed)
    b = make_geometry(pulses=pulses, samples=samples, width=width, length=length,
                      spacing=spacing, centre_height=1000.0, quantise=quantise, **kw)
    b.dem = volcano_dem(rng, length, width)
    return b


def mini_samples(seed: int, pulses: int, samples: int) -> np.ndarray:
    """Integer-valued complex64 samples (components k/16, |k| <= 64), exactly
    reproducible on any platform from the seed."""
    rng = np.random.default_rng([seed, 2])
    raw = rng.integers(-64, 65, size=(pulses, samples, 2), dtype=np.int32).astype(np.float32)
    return (raw[..., 0] + 1j * raw[..., 1]).astype(np.complex64) * np.float32(1.0 / 16)


def mini_fixture(seed: int, pulses: int = 320, samples: int = 384, width: int = 48,
                 length: int = 40, spacing: float = 0.0002, aperture: int = 96,
                 angc0: float = 0.0, angc1: float = 0.0, dem_kind: str = "slope",
                 latlons_inset: int = 0) -> Burst:
    """Small scene for the golden fixtures: integer-valued samples
    (``mini_samples``) and an integer DEM, so that everything but the orbit
    arrays can be regenerated bit for bit; the fixtures store the orbit
    arrays themselves."""
    rng = np.random.default_rng([seed, 1])
    b = make_geometry(pulses=pulses, samples=samples, width=width, length=length,
                      spacing=spacing, centre_height=200.0, aperture=aperture,
                      angc0=angc0, angc1=angc1)
    if dem_kind == "flat":
        b.dem = np.full((length, width), 200, np.int16)
    else:
        yy, xx = np.mgrid[0:length, 0:width]
        b.dem = (150 + 3 * xx + 2 * yy + rng.integers(-20, 21, (length, width))).astype(np.int16)
    b.burst = mini_samples(seed, pulses, samples)
    if latlons_inset:
        # shrink the pixel box: firstpix = inset, lastpix = W - 1 - inset
        b.latlons[2] = b.firstlon + (latlons_inset + 0.25) * b.deltalon
        b.latlons[3] = b.firstlon + (width - 1 - latlons_inset + 0.25) * b.deltalon
    return b


def host_clutter_samples(b: Burst, seed: int, ntargets: int = 200, target_db: float = 30.0,
                         samples: Optional[int] = None) -> None:
    """Fill b.burst on the host with circular complex Gaussian clutter (unit
    power per sample) plus `ntargets` point targets at +`target_db` on random
    grid pixels of the burst's pixel window (``add_point_targets``): the
    statistics of the device workloads' range lines, drawn with numpy so that
    CPU-only runs need neither a GPU nor the CUDA library.  `samples`
    (default b.samples) sets the line length."""
    rng = np.random.default_rng([seed, 7])
    P = b.rawdatalines
    S = b.samples if samples is None else samples
    z = rng.standard_normal((P, S, 2), dtype=np.float32) * np.float32(math.sqrt(0.5))
    b.burst = (z[..., 0] + 1j * z[..., 1]).astype(np.complex64)
    del z
    ll = int((b.latlons[0] - b.firstlat) / b.deltalat)
    fl = int((b.latlons[1] - b.firstlat) / b.deltalat)
    fl, ll = min(max(fl, 0), b.demlength - 1), min(max(ll, 0), b.demlength - 1)
    fp = max(int((b.latlons[2] - b.firstlon) / b.deltalon), 0)
    lp = min(int((b.latlons[3] - b.firstlon) / b.deltalon), b.demwidth - 1)
    lines = rng.integers(fl, ll + 1, ntargets)
    pix = rng.integers(fp, lp + 1, ntargets)
    h = b.dem[lines, pix].astype(np.float64) if b.dem is not None else np.zeros(ntargets)
    add_point_targets(b, grid_ecef(b, lines, pix, h), np.full(ntargets, 10.0 ** (target_db / 20.0)))


# Sentinel-1 header fields the burst-parameter derivation reads (byte
# offsets in a line's 80-byte header, sentinel/backprojectgpusub.f90:266-299,
# 406-429): range decimation code (40), rank (49, low 5 bits), PRI code (50,
# 24-bit big endian, in units of 1/fref us), SWST code (53, idem), azimuth
# beam word (60, 16-bit big endian, address in the low 10 bits), line time
# (68, native double).
FREF_MHZ = 37.53472224


def encode_line_headers(times, pri_code: int, rank: int, swst_code: int, decimation: int,
                        beam_address) -> np.ndarray:
    """[P][10] complex64 holding each line's 80-byte header with the given
    fields (the other bytes zero): the first 10 samples of a decoded line."""
    times = np.asarray(times, np.float64)
    P = times.shape[0]
    beam = np.broadcast_to(np.asarray(beam_address, np.int64), (P,))
    h = np.zeros((P, 80), np.uint8)
    h[:, 40] = decimation & 255
    h[:, 49] = rank & 31
    for off, v in ((50, pri_code), (53, swst_code)):
        h[:, off] = (v >> 16) & 255
        h[:, off + 1] = (v >> 8) & 255
        h[:, off + 2] = v & 255
    h[:, 60] = (beam >> 8) & 3
    h[:, 61] = beam & 255
    h[:, 68:76] = times.astype("<f8").view(np.uint8).reshape(P, 8)
    return h.view(np.complex64).reshape(P, 10)


def header_codes(prf: float, rngstart: float, rank: int = 9):
    """PRI and SWST codes whose decoded PRF and near range come closest to
    the given ones (the inverse of burstparams, up to the codes' rounding)."""
    pri_us = 1e6 / prf
    pri_code = int(round(pri_us * FREF_MHZ))
    pri = pri_code / FREF_MHZ * 1e-6
    swst = 2.0 * (rngstart - 60.0) / C_LIGHT - rank * pri
    return pri_code, int(round(swst * 1e6 * FREF_MHZ))


# Fields of a Burst that a fixture stores verbatim.
ARRAY_FIELDS = ("satloc", "satvel", "pulse_time", "latlons", "timeorbit", "xx", "vv", "xyz_mid",
                "vel_mid", "dem")
FLOAT_FIELDS = ("deltalat", "deltalon", "firstlat", "firstlon", "rngstart", "rngend", "tstart",
                "tend", "tmid", "dtaz", "dmrg", "wvl", "angc0", "angc1", "prf")
INT_FIELDS = ("demwidth", "demlength", "aperture", "iaperture")


def burst_to_arrays(b: Burst) -> dict:
    out = {k: np.asarray(getattr(b, k)) for k in ARRAY_FIELDS}
    out["floats"] = np.array([getattr(b, k) for k in FLOAT_FIELDS], np.float64)
    out["ints"] = np.array([getattr(b, k) for k in INT_FIELDS] + list(b.burst.shape), np.int64)
    return out


def burst_from_arrays(a, samples: np.ndarray) -> Burst:
    kw = {k: np.array(a[k]) for k in ARRAY_FIELDS if k != "dem"}
    kw.update({k: float(v) for k, v in zip(FLOAT_FIELDS, a["floats"])})
    ints = [int(v) for v in a["ints"]]
    kw.update({k: v for k, v in zip(INT_FIELDS, ints[:len(INT_FIELDS)])})
    b = Burst(burst=samples, **kw)
    b.dem = np.array(a["dem"], np.int16)
    return b


# --------------------------------------------------------------------------
# multi-burst scenes


@dataclasses.dataclass
class SceneGrid:
    """A shared lat/lon grid and DEM for several bursts."""
    firstlat: float
    firstlon: float
    spacing: float
    width: int
    length: int
    dem: np.ndarray  # [length][width] int16


def _burst_on_grid(grid: SceneGrid, orbit: CircularOrbit, tmid: float, pulses: int, samples: int,
                   near_range: float, window, aperture: Optional[int] = None, wvl=WAVELENGTH,
                   prf=PRF, fs=RANGE_FS) -> Burst:
    """One burst of `pulses` lines centred at time tmid, whose latlons select
    the pixel window ((line0, line1), (pix0, pix1)) of the shared grid."""
    dtaz = 1.0 / prf
    tstart = tmid - 0.5 * (pulses - 1) * dtaz
    tend = tstart + (pulses - 1) * dtaz
    t0 = math.floor((tstart - 30.0) / SV_SPACING) * SV_SPACING + SV_SPACING
    timeorbit = t0 + SV_SPACING * np.arange(11, dtype=np.float64)
    xx, vv = orbit.state(timeorbit)
    ptime = tstart + np.arange(pulses, dtype=np.float64) * dtaz
    sx, sv = interp_pulses(timeorbit, xx, vv, ptime)
    sx, sv = quantise_positions(sx, sv)
    xyz_mid, vel_mid = intp_orbit(timeorbit, xx, vv, 0.5 * (tstart + tend))
    dmrg = C_LIGHT / 2.0 / fs
    (l0, l1), (p0, p1) = window
    sp = grid.spacing
    latlons = np.array([grid.firstlat - (l1 + 0.25) * sp, grid.firstlat - (l0 + 0.25) * sp,
                        grid.firstlon + (p0 + 0.25) * sp, grid.firstlon + (p1 + 0.25) * sp])
    b = Burst(
        burst=np.zeros((0, samples), np.complex64), satloc=np.ascontiguousarray(sx),
        satvel=np.ascontiguousarray(sv), pulse_time=ptime, demwidth=grid.width,
        demlength=grid.length, deltalat=-sp, deltalon=sp, firstlat=grid.firstlat,
        firstlon=grid.firstlon, latlons=latlons, timeorbit=timeorbit,
        xx=np.ascontiguousarray(xx), vv=np.ascontiguousarray(vv), rngstart=near_range,
        rngend=near_range + (samples - 1) * dmrg, tstart=tstart, tend=tend,
        tmid=0.5 * (tstart + tend), xyz_mid=np.ascontiguousarray(xyz_mid),
        vel_mid=np.ascontiguousarray(vel_mid), dtaz=dtaz, dmrg=dmrg, wvl=wvl,
        aperture=aperture if aperture is not None else aperture_points(sv, near_range, wvl, prf),
        iaperture=0, angc0=0.0, angc1=0.0, prf=prf)
    b.dem = grid.dem
    b.pulses = pulses
    return b


def iw_scene(seed: int = 1003, nswaths: int = 3, nbursts: int = 9,
             samples=(18000, 21500, 25600), near=(800.0e3, 838.0e3, 884.0e3),
             pulses=(1380, 1620), widths=(2000, 2600), lengths=(1000, 1300),
             spacing: float = 1e-4, burst_step_s: float = 0.45, lat0: float = 19.4,
             dem_kind: str = "volcano", device=None):
    """Configuration 3: a full IW scene -- `nswaths` subswaths x `nbursts`
    bursts of uneven size (P uniform in `pulses`, S per subswath), each mapped
    to its own overlapping sub-grid (W in `widths`, L in `lengths`) of one
    shared grid and DEM.  Returns (SceneGrid, [Burst]) in acquisition order
    (burst-major, subswath-minor).  Burst samples are left empty (shape
    [0][S]); the workload builder fills them on the device.  With a torch
    `device` the DEM is synthesised there (grid.dem is then a device tensor)."""
    rng = np.random.default_rng(seed)
    inc = math.radians(ORBIT_INCL_DEG)
    T0 = 43200.25
    u0 = math.asin(math.sin(math.radians(lat0)) / math.sin(inc))
    orbit = CircularOrbit(u0=u0, epoch=T0)
    dmrg = C_LIGHT / 2.0 / RANGE_FS
    plan = []
    for ib in range(nbursts):
        for isw in range(nswaths):
            tm = T0 + (ib - (nbursts - 1) / 2.0) * burst_step_s
            P = int(rng.integers(pulses[0], pulses[1] + 1))
            S = int(samples[isw])
            r0 = float(near[isw])
            smid, vmid = orbit.state(np.array([tm]))
            pc = zero_doppler_point(smid[0], vmid[0], r0 + 0.5 * (S - 1) * dmrg, 1000.0)
            clat, clon, _ = ecef_to_llh(pc)
            W = int(rng.integers(widths[0], widths[1] + 1))
            L = int(rng.integers(lengths[0], lengths[1] + 1))
            plan.append((tm, P, S, r0, float(clat), float(clon), W, L))
    lat_hi = max(p[4] + 0.5 * p[7] * spacing for p in plan) + 20 * spacing
    lat_lo = min(p[4] - 0.5 * p[7] * spacing for p in plan) - 20 * spacing
    lon_lo = min(p[5] - 0.5 * p[6] * spacing for p in plan) - 20 * spacing
    lon_hi = max(p[5] + 0.5 * p[6] * spacing for p in plan) + 20 * spacing
    length = int(math.ceil((lat_hi - lat_lo) / spacing)) + 1
    width = int(math.ceil((lon_hi - lon_lo) / spacing)) + 1
    if dem_kind == "volcano" and device is not None:
        dem = volcano_dem_torch(int(rng.integers(2**31)), length, width, device, radius_frac=0.35)
    elif dem_kind == "volcano":
        dem = volcano_dem(rng, length, width, radius_frac=0.35)
    else:
        dem = np.full((length, width), 1000, np.int16)
    grid = SceneGrid(firstlat=lat_hi, firstlon=lon_lo, spacing=spacing, width=width,
                     length=length, dem=dem)
    bursts = []
    for tm, P, S, r0, clat, clon, W, L in plan:
        cl = int(round((grid.firstlat - clat) / spacing))
        cp = int(round((clon - grid.firstlon) / spacing))
        l0 = max(0, cl - L // 2)
        p0 = max(0, cp - W // 2)
        win = ((l0, min(length - 1, l0 + L - 1)), (p0, min(width - 1, p0 + W - 1)))
        bursts.append(_burst_on_grid(grid, orbit, tm, P, S, r0, win))
    return grid, bursts


def mini_scene(seed: int = 21, width: int = 64, length: int = 60, spacing: float = 0.0002):
    """Three small bursts on one shared grid, for tests: consecutive in time
    (overlapping output windows), uneven pulse and sample counts (one odd),
    integer-valued samples (``mini_samples``).  Returns (SceneGrid, [Burst])."""
    rng = np.random.default_rng([seed, 3])
    inc = math.radians(ORBIT_INCL_DEG)
    T0 = 43200.25
    orbit = CircularOrbit(u0=math.asin(math.sin(math.radians(19.4)) / math.sin(inc)), epoch=T0)
    dmrg = C_LIGHT / 2.0 / RANGE_FS
    smid, vmid = orbit.state(np.array([T0]))
    pc = zero_doppler_point(smid[0], vmid[0], 800.0e3, 200.0)
    clat, clon, _ = ecef_to_llh(pc)
    grid = SceneGrid(firstlat=float(clat) + 0.5 * (length - 1) * spacing,
                     firstlon=float(clon) - 0.5 * (width - 1) * spacing, spacing=spacing,
                     width=width, length=length,
                     dem=(150 + 2 * np.arange(width)[None, :] + np.arange(length)[:, None] +
                          rng.integers(-15, 16, (length, width))).astype(np.int16))
    specs = [(-0.05, 300, 384, ((4, 40), (3, 58))), (0.0, 320, 401, ((14, 50), (6, 63))),
             (0.05, 280, 416, ((22, 59), (0, 55)))]
    bursts = []
    for i, (dt, P, S, win) in enumerate(specs):
        b = _burst_on_grid(grid, orbit, T0 + dt, P, S, 800.0e3 - 0.5 * (S - 1) * dmrg, win,
                           aperture=96)
        b.burst = mini_samples(seed * 10 + i, P, S)
        b.pulses = 0
        bursts.append(b)
    return grid, bursts
