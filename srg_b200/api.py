"""Python entry points of the backprojection library.

* ``azimuth_compress_files``: the reference-facing call -- the 33-argument
  by-reference ``azimuth_compress_`` of libsrg_bp.so, exactly as
  sentinel/backprojectgpusub.f90:244-247 makes it, on a DEM file and a .geo
  file.
* ``DeviceBurst`` / ``backproject``: device-resident bursts (torch tensors
  for memory and streams) through ``srg_bp_bursts_device``, one persistent
  launch for any number of bursts.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import FORM_FP64, FORM_SPLIT, BurstDesc, check, default_options, lib
from .scene import Burst

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def limits(b: Burst):
    """Reference line/pixel limits (sentinel/azimuth_compress.cu:295-301, 378-379)."""
    ll = int((b.latlons[0] - b.firstlat) / b.deltalat)
    fl = int((b.latlons[1] - b.firstlat) / b.deltalat)
    fl = min(max(fl, 0), b.demlength - 1)
    ll = min(max(ll, 0), b.demlength - 1)
    fp = max(int((b.latlons[2] - b.firstlon) / b.deltalon), 0)
    lp = min(int((b.latlons[3] - b.firstlon) / b.deltalon), b.demwidth)
    return fl, ll, fp, lp


def azimuth_compress_files(b: Burst, fdout: int, fddem: int, burst: Optional[np.ndarray] = None):
    """Call the drop-in ``azimuth_compress_`` (33 by-reference arguments)."""
    prepare_azimuth_compress(b, fdout, fddem, burst)()


def prepare_azimuth_compress(b: Burst, fdout: int, fddem: int, burst: Optional[np.ndarray] = None):
    """The 33 by-reference arguments of one ``azimuth_compress_`` call, built
    once; returns a callable that makes the call (as a Fortran caller does, with
    its arrays and scalars already in place)."""
    L = lib()
    burst = np.ascontiguousarray(b.burst if burst is None else burst, np.complex64)
    keep = {k: _d(getattr(b, k)) for k in
            ("satloc", "latlons", "timeorbit", "xx", "vv", "xyz_mid", "vel_mid", "pulse_time")}
    i = {k: C.c_int(v) for k, v in dict(P=b.rawdatalines, S=b.samples, W=b.demwidth,
                                        L=b.demlength, fo=fdout, fd=fddem, n=b.numstatevec,
                                        ap=b.aperture, iap=b.iaperture).items()}
    d = {k: C.c_double(getattr(b, k)) for k in
         ("deltalat", "deltalon", "firstlat", "firstlon", "rngstart", "rngend", "tstart", "tend",
          "tmid", "dtaz", "dmrg", "wvl", "angc0", "angc1", "prf")}
    r = C.byref
    p = lambda a: a.ctypes.data_as(_dp)  # noqa: E731
    args = (
        burst.ctypes.data_as(_fp), p(keep["satloc"]), r(i["P"]), r(i["S"]), r(i["W"]), r(i["L"]),
        r(i["fo"]), r(i["fd"]), r(d["deltalat"]), r(d["deltalon"]), r(d["firstlat"]),
        r(d["firstlon"]), p(keep["latlons"]), p(keep["timeorbit"]), p(keep["xx"]), p(keep["vv"]),
        r(i["n"]), r(d["rngstart"]), r(d["rngend"]), r(d["tstart"]), r(d["tend"]), r(d["tmid"]),
        p(keep["xyz_mid"]), p(keep["vel_mid"]), p(keep["pulse_time"]), r(d["dtaz"]), r(d["dmrg"]),
        r(d["wvl"]), r(i["ap"]), r(i["iap"]), r(d["angc0"]), r(d["angc1"]), r(d["prf"]))
    fn = L.azimuth_compress_
    held = (burst, keep, i, d)  # the buffers the pointers refer to stay alive with the call

    def call():
        fn(*args)
        return held is not None
    return call


def azimuth_compress_status(b: Burst, fdout: int, fddem: int, form: int = FORM_SPLIT,
                            tile_cfg: int = -1, burst: Optional[np.ndarray] = None,
                            **options) -> int:
    """The status-returning twin of the drop-in entry (raises on error);
    `options`: further srg_bp_options fields (spin_limit, scratch_limit, ...)."""
    L = lib()
    burst = np.ascontiguousarray(b.burst if burst is None else burst, np.complex64)
    keep = {k: _d(getattr(b, k)) for k in
            ("satloc", "latlons", "timeorbit", "xx", "vv", "xyz_mid", "vel_mid")}
    p = lambda a: a.ctypes.data_as(_dp)  # noqa: E731
    o = default_options(form, tile_cfg)
    for k, v in options.items():
        setattr(o, k, v)
    rc = L.srg_azimuth_compress(
        burst.ctypes.data_as(_fp), p(keep["satloc"]), b.rawdatalines, b.samples, b.demwidth,
        b.demlength, fdout, fddem, b.deltalat, b.deltalon, b.firstlat, b.firstlon,
        p(keep["latlons"]), p(keep["timeorbit"]), p(keep["xx"]), p(keep["vv"]), b.numstatevec,
        b.rngstart, b.rngend, b.tmid, p(keep["xyz_mid"]), p(keep["vel_mid"]), b.dmrg, b.wvl,
        b.aperture, b.angc0, b.angc1, b.prf, C.byref(o))
    check(rc)
    return rc


def interp_error(lines, nsamps: Optional[int] = None, sample_lines: int = 64, stream=None):
    """(linear, 2x-oversampled) expected RMS phase error (rad) of the range
    interpolation on device lines ([nlines][ld] complex64 tensor)."""
    el, eo = C.c_double(), C.c_double()
    nsamps = lines.shape[1] if nsamps is None else nsamps
    check(lib().srg_interp_error(C.c_void_p(lines.data_ptr()), lines.stride(0), lines.shape[0],
                                 nsamps, sample_lines, C.byref(el), C.byref(eo),
                                 C.c_void_p(_stream_ptr(stream))))
    return float(el.value), float(eo.value)


def dropin_flush(device: int = -1) -> None:
    """Wait for the overlapped drop-in calls of `device` (-1: every device) to
    finish their merges; raises the first failure among them not yet
    reported."""
    check(lib().srg_dropin_flush(device))


def dropin_last_bytes(device: int = -1):
    """(host-to-device, device-to-host) bytes of the last drop-in call."""
    h, d = C.c_longlong(), C.c_longlong()
    check(lib().srg_dropin_last_bytes(device, C.byref(h), C.byref(d)))
    return int(h.value), int(d.value)


def burst_params(lines: np.ndarray, satvel: np.ndarray) -> dict:
    """Per-burst scalars of the azimuth_compress_ call (srg_burst_params:
    burstparams, fdopcoefs, aperture and limits of
    sentinel/backprojectgpusub.f90) from decoded lines whose first 10 samples
    still hold the line headers ([P][S] complex64, host) and the per-pulse
    velocities ([P][3])."""
    lines = np.ascontiguousarray(lines, np.complex64)
    sv = _d(satvel)
    r = _lib.BurstParams()
    check(lib().srg_burst_params(C.c_void_p(lines.ctypes.data), lines.shape[1], lines.shape[0],
                                 lines.shape[1], sv.ctypes.data_as(_dp), C.byref(r)))
    return {k: getattr(r, k) for k, _ in r._fields_ if k != "pad"}


def set_default_form(form: int, tile_cfg: int = -1, overlap: Optional[int] = None) -> None:
    """Options of azimuth_compress_ (srg_set_default_options): form, shape and,
    when given, whether calls overlap (else the environment's default)."""
    o = default_options(form, tile_cfg)
    if overlap is not None:
        o.overlap = int(overlap)
    lib().srg_set_default_options(C.byref(o))


@dataclasses.dataclass
class DeviceBurst:
    """A burst resident in device memory (torch tensors) plus its descriptor."""

    b: Burst
    burst: "object"        # torch complex64 [P][S] (or a view with row stride ldb)
    satloc: "object"       # torch float64 [P][3]
    dem: "object"          # torch int16 [nlines][W] (rows firstline.. of the grid)
    out: "object"          # torch complex64 [nlines][W]
    firstline: int
    nlines: int
    firstpix: int
    lastpix: int
    out_pix0: int = 0      # grid pixel of out[:, 0]
    keep: dict = dataclasses.field(default_factory=dict)

    def desc(self, coef_ptr: int = 0) -> BurstDesc:
        b = self.b
        d = BurstDesc()
        d.burst = self.burst.data_ptr()
        d.satloc = self.satloc.data_ptr()
        d.dem = self.dem.data_ptr()
        d.out = self.out.data_ptr()
        d.coef = coef_ptr or None
        d.ldb = self.burst.stride(0)
        d.dem_ld = self.dem.stride(0)
        d.out_ld = self.out.stride(0)
        d.P = b.rawdatalines
        d.S = b.samples
        d.demwidth = b.demwidth
        d.firstline, d.nlines, d.firstpix, d.lastpix = (self.firstline, self.nlines, self.firstpix,
                                                        self.lastpix)
        d.out_pix0 = self.out_pix0
        d.aperture = b.aperture
        d.firstlat, d.deltalat, d.firstlon, d.deltalon = b.firstlat, b.deltalat, b.firstlon, b.deltalon
        d.rngstart, d.rngend, d.dmrg, d.wvl = b.rngstart, b.rngend, b.dmrg, b.wvl
        for k in ("timeorbit", "xx", "vv"):
            self.keep[k] = _d(getattr(b, k))
            setattr(d, k, self.keep[k].ctypes.data_as(_dp))
        d.numstatevec = b.numstatevec
        d.tmid = b.tmid
        for i in range(3):
            d.xyz_mid[i] = float(b.xyz_mid[i])
            d.vel_mid[i] = float(b.vel_mid[i])
        d.angc0, d.angc1, d.prf = b.angc0, b.angc1, b.prf
        return d


def to_device(b: Burst, device="cuda", burst_tensor=None, dem_tensor=None,
              narrow_out: bool = False) -> DeviceBurst:
    """Device copy of a burst.  dem_tensor: an already-resident full DEM
    ([demlength][demwidth] int16) to take the slab from without copying;
    narrow_out: output columns only for [firstpix, min(lastpix, W-1)]."""
    import torch

    fl, ll, fp, lp = limits(b)
    nl = ll - fl + 1
    if burst_tensor is None:
        burst_tensor = torch.from_numpy(np.ascontiguousarray(b.burst, np.complex64)).to(device)
    sat = torch.from_numpy(_d(b.satloc)).to(device)
    if dem_tensor is not None:
        dem = dem_tensor[fl:fl + nl]
    else:
        dem = torch.from_numpy(np.ascontiguousarray(b.dem[fl:fl + nl], np.int16)).to(device)
    if narrow_out:
        ncols = max(0, min(lp, b.demwidth - 1) - fp + 1)
        out = torch.zeros((nl, max(ncols, 1)), dtype=torch.complex64, device=device)
        pix0 = fp
    else:
        out = torch.zeros((nl, b.demwidth), dtype=torch.complex64, device=device)
        pix0 = 0
    return DeviceBurst(b=b, burst=burst_tensor, satloc=sat, dem=dem, out=out, firstline=fl,
                       nlines=nl, firstpix=fp, lastpix=lp, out_pix0=pix0)


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(stream)


def backproject(bursts: Sequence[DeviceBurst], form: int = FORM_SPLIT, tile_cfg: int = -1,
                stream=None, sync: bool = True, coefs=None, tile_shear: Optional[int] = None) -> None:
    """Backproject device bursts into their `out` tensors (one launch).
    coefs: optional per-burst device tensors of azimuth-centre parabolas
    ([nlines][3] float64, from ``line_centres``); without them the centres are
    solved on the device first.  tile_shear: srg_bp_options.tile_shear (None:
    chosen from each burst's geometry)."""
    ptrs = [c.data_ptr() for c in coefs] if coefs is not None else [0] * len(bursts)
    arr = (BurstDesc * len(bursts))(*[db.desc(p) for db, p in zip(bursts, ptrs)])
    o = default_options(form, tile_cfg)
    if tile_shear is not None:
        o.tile_shear = int(tile_shear)
    st = _stream_ptr(stream)
    check(lib().srg_bp_bursts_device(arr, len(bursts), C.byref(o), C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))


def count_terms(bursts: Sequence[DeviceBurst], stream=None) -> int:
    arr = (BurstDesc * len(bursts))(*[db.desc() for db in bursts])
    n = C.c_int64()
    check(lib().srg_count_terms_device(arr, len(bursts), C.byref(n), C.c_void_p(_stream_ptr(stream))))
    return int(n.value)


def line_centres(db: DeviceBurst, stream=None, out=None, sync: bool = True):
    """Per-line azimuth-centre parabolas of a device burst ([nlines][3] float64)."""
    import torch
    coef = out if out is not None else torch.zeros((db.nlines, 3), dtype=torch.float64,
                                                   device=db.out.device)
    d = db.desc()
    st = _stream_ptr(stream)
    check(lib().srg_line_centres_device(C.byref(d), C.c_void_p(coef.data_ptr()), C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))
    return coef


def pulse_orbit(times, b: Burst, stream=None):
    """Per-pulse Hermite orbit on the device; times: torch float64 [P] (device)."""
    import torch
    P = times.shape[0]
    pos = torch.empty((P, 3), dtype=torch.float64, device=times.device)
    vel = torch.empty_like(pos)
    to, xx, vv = _d(b.timeorbit), _d(b.xx), _d(b.vv)
    check(lib().srg_pulse_orbit_device(
        C.c_void_p(times.data_ptr()), P, to.ctypes.data_as(_dp), xx.ctypes.data_as(_dp),
        vv.ctypes.data_as(_dp), len(to), C.c_void_p(pos.data_ptr()), C.c_void_p(vel.data_ptr()),
        C.c_void_p(_stream_ptr(stream))))
    return pos, vel


def merge(dst, src, stream=None) -> None:
    """dst[r][c] = src[r][c] where |Re(src)| > 1e-18 (the reference merge rule)."""
    rows, cols = src.shape
    check(lib().srg_merge_device(C.c_void_p(dst.data_ptr()), dst.stride(0),
                                 C.c_void_p(src.data_ptr()), src.stride(0), rows, cols,
                                 C.c_void_p(_stream_ptr(stream))))


def forward_project(db: DeviceBurst, refl, satvel, antenna: float = 10.0, stream=None,
                    range_offset=None) -> None:
    """Accumulate the echo of a per-pixel reflectivity field into db.burst;
    range_offset: optional float32 tensor of the same shape as refl (metres
    added to each scatterer's range)."""
    d = db.desc()
    ro = 0
    if range_offset is not None:
        if range_offset.shape != refl.shape or range_offset.stride(0) != refl.stride(0):
            raise ValueError("range_offset must match refl's shape and row stride")
        ro = range_offset.data_ptr()
    check(lib().srg_forward_project_device(C.byref(d), C.c_void_p(refl.data_ptr()), refl.stride(0),
                                           C.c_void_p(satvel.data_ptr()), antenna, C.c_void_p(ro),
                                           C.c_void_p(_stream_ptr(stream))))


def _xm_check(t, na):
    import torch
    if t.dtype != torch.complex64 or t.dim() != 2 or t.stride(1) != 1 or not t.is_cuda:
        raise ValueError("images must be 2-D complex64 CUDA tensors with unit column stride")


def crossmul(slc1, slc2, looksac: int = 1, looksdn: Optional[int] = None, scale: float = 1.0,
             mask: bool = True, nvalid: Optional[int] = None, stream=None, sync: bool = True):
    """Interferogram and amplitude images of two co-registered device images
    (srg_crossmul_device; the reference's int/crossmul.f90).  Returns
    (igram, amp), complex64 [nvalid // looksdn][na // looksac] on the device."""
    import torch
    looksdn = looksac if looksdn is None else looksdn
    nd, na = slc1.shape
    nvalid = nd if nvalid is None else nvalid
    for t in (slc1, slc2):
        _xm_check(t, na)
    if slc2.shape != slc1.shape or slc2.stride(0) != slc1.stride(0):
        raise ValueError("images must have the same shape and row stride")
    shape = (nvalid // looksdn, na // looksac)
    ig = torch.empty(shape, dtype=torch.complex64, device=slc1.device)
    am = torch.empty_like(ig)
    st = _stream_ptr(stream)
    check(lib().srg_crossmul_device(
        C.c_void_p(slc1.data_ptr()), C.c_void_p(slc2.data_ptr()), slc1.stride(0), na, nvalid,
        looksac, looksdn, scale, int(bool(mask)), C.c_void_p(ig.data_ptr()), C.c_void_p(am.data_ptr()),
        C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))
    return ig, am


def crossmul_stack(slcs, looksac: int = 1, looksdn: Optional[int] = None, scale: float = 1.0,
                   mask: bool = True, stream=None, sync: bool = True, outs=None):
    """Interferograms of the sequential pairs (k, k+1) of a list of device
    images (srg_crossmul_stack_device: each image transformed once).
    Returns ([igram_k], [amp_k]); `outs` may supply them."""
    import torch
    looksdn = looksac if looksdn is None else looksdn
    nd, na = slcs[0].shape
    for t in slcs:
        _xm_check(t, na)
        if t.shape != slcs[0].shape or t.stride(0) != slcs[0].stride(0):
            raise ValueError("images must have the same shape and row stride")
    shape = (nd // looksdn, na // looksac)
    if outs is None:
        igs = [torch.empty(shape, dtype=torch.complex64, device=slcs[0].device) for _ in slcs[1:]]
        ams = [torch.empty_like(g) for g in igs]
    else:
        igs, ams = outs
    n = len(slcs)
    pin = (C.c_void_p * n)(*[t.data_ptr() for t in slcs])
    pig = (C.c_void_p * (n - 1))(*[t.data_ptr() for t in igs])
    pam = (C.c_void_p * (n - 1))(*[t.data_ptr() for t in ams])
    st = _stream_ptr(stream)
    check(lib().srg_crossmul_stack_device(pin, n, slcs[0].stride(0), na, nd, looksac, looksdn, scale,
                                          int(bool(mask)), pig, pam, C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))
    return igs, ams


def range_replica(samplefreq: float, startfreq: float, ramprate: float, pulselength: float,
                  n: int = 32768):
    """The reference's chirp replica (complex64 [n], zero-padded) and npts."""
    rep = np.zeros(n, np.complex64)
    npts = C.c_int()
    check(lib().srg_range_replica(samplefreq, startfreq, ramprate, pulselength,
                                  C.c_void_p(rep.ctypes.data), n, C.byref(npts)))
    return rep, int(npts.value)


def range_compress(lines, samplefreq: float, startfreq: float, ramprate: float, pulselength: float,
                   nsamps: Optional[int] = None, out=None, stream=None, sync: bool = True):
    """Range-compress decoded echo lines (complex64 CUDA tensor [nlines][>= nsamps],
    line headers stripped) with the chirp of the given pulse parameters
    (srg_range_compress_device).  Returns the [nlines][nvalid] complex64 tensor
    (or writes into `out`, whose rows must hold nvalid samples)."""
    import torch
    if lines.dtype != torch.complex64 or lines.dim() != 2 or lines.stride(1) != 1 or not lines.is_cuda:
        raise ValueError("lines must be a 2-D complex64 CUDA tensor with unit column stride")
    nlines = lines.shape[0]
    nsamps = lines.shape[1] if nsamps is None else nsamps
    _, npts = range_replica(samplefreq, startfreq, ramprate, pulselength)
    nvalid = nsamps - npts
    if out is None:
        out = torch.empty((nlines, max(nvalid, 1)), dtype=torch.complex64, device=lines.device)
    nv = C.c_int()
    st = _stream_ptr(stream)
    check(lib().srg_range_compress_device(C.c_void_p(lines.data_ptr()), lines.stride(0), nlines, nsamps,
                                          samplefreq, startfreq, ramprate, pulselength,
                                          C.c_void_p(out.data_ptr()), out.stride(0), C.byref(nv),
                                          C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))
    return out


def oversample_taps():
    """The 4 half-sample taps (each used on both sides) of srg_oversample_range_device."""
    h = np.zeros(4, np.float32)
    lib().srg_oversample_taps(C.c_void_p(h.ctypes.data))
    return h


def oversample2(db: DeviceBurst, stream=None, sync: bool = True) -> DeviceBurst:
    """A copy of a device burst with its range lines oversampled 2x
    (srg_oversample_range_device) and the burst geometry adjusted: 2S - 1
    samples at dmrg / 2 over the same [rngstart, rngend].  The copy shares the
    satloc, DEM and output tensors of `db`."""
    import copy
    import torch
    P, S = db.b.rawdatalines, db.b.samples
    ld = 2 * S  # even row length keeps each row 16-byte aligned for TMA
    out = torch.empty((P, ld), dtype=torch.complex64, device=db.burst.device)
    st = _stream_ptr(stream)
    check(lib().srg_oversample_range_device(C.c_void_p(db.burst.data_ptr()), db.burst.stride(0), P, S,
                                            C.c_void_p(out.data_ptr()), ld, C.c_void_p(st)))
    if sync:
        check(lib().srg_sync_check(C.c_void_p(st)))
    b2 = copy.copy(db.b)
    b2.pulses = P
    b2.burst = np.zeros((0, 2 * S - 1), np.complex64)  # shape only: the samples live on the device
    b2.dmrg = db.b.dmrg / 2.0
    return DeviceBurst(b=b2, burst=out[:, :2 * S - 1], satloc=db.satloc, dem=db.dem, out=db.out,
                       firstline=db.firstline, nlines=db.nlines, firstpix=db.firstpix,
                       lastpix=db.lastpix, out_pix0=db.out_pix0)


class Scene:
    """A reusable plan over device bursts (srg_scene_*): azimuth centres,
    one persistent backprojection launch for all bursts and the ordered merge
    into `raster` (optional, [lines][cols] complex64 on the device), replayed
    from a CUDA graph on a non-default stream."""

    def __init__(self, bursts: Sequence[DeviceBurst], raster=None, form: int = FORM_SPLIT,
                 tile_cfg: int = -1, tile_shear: Optional[int] = None):
        self.bursts = list(bursts)
        self.raster = raster
        self._descs = (BurstDesc * len(self.bursts))(*[db.desc() for db in self.bursts])
        o = default_options(form, tile_cfg)
        if tile_shear is not None:
            o.tile_shear = int(tile_shear)
        h = C.c_void_p()
        if raster is not None:
            args = (C.c_void_p(raster.data_ptr()), raster.stride(0), raster.shape[0], raster.shape[1])
        else:
            args = (None, 0, 0, 0)
        check(lib().srg_scene_create(self._descs, len(self.bursts), *args, C.byref(o), C.byref(h)))
        self.handle = h

    def run(self, stream=None) -> None:
        check(lib().srg_scene_run(self.handle, C.c_void_p(_stream_ptr(stream))))

    def run_stages(self, stages: int, stream=None) -> None:
        """1 = azimuth centres, 2 = backprojection, 4 = merge (no graph)."""
        check(lib().srg_scene_run_stages(self.handle, stages, C.c_void_p(_stream_ptr(stream))))

    def sync(self, stream=None) -> None:
        check(lib().srg_scene_sync(self.handle, C.c_void_p(_stream_ptr(stream))))

    def terms(self) -> int:
        n = C.c_int64()
        check(lib().srg_scene_terms(self.handle, C.byref(n)))
        return int(n.value)

    def tune(self, iters: int = 3):
        cfg, ms = C.c_int(), C.c_double()
        check(lib().srg_scene_tune(self.handle, iters, C.byref(cfg), C.byref(ms)))
        return int(cfg.value), float(ms.value)

    def autotune(self, interp_budget: float = 0.0, iters: int = 3, use_cache: bool = True) -> dict:
        """srg_scene_autotune: the interpolation within `interp_budget` (RMS
        phase error in rad; 0 keeps the plan's), then the fastest shape
        (or the cached one).  Returns the srg_tune_result fields."""
        q = _lib.TuneRequest(iters, int(bool(use_cache)), float(interp_budget))
        r = _lib.TuneResult()
        check(lib().srg_scene_autotune(self.handle, C.byref(q), C.byref(r)))
        return {k: getattr(r, k) for k, _ in r._fields_}

    def set_interp(self, interp: int) -> None:
        check(lib().srg_scene_set_interp(self.handle, interp))

    def interp(self) -> int:
        return int(lib().srg_scene_interp(self.handle))

    def set_form(self, form: int, tile_cfg: int = -1) -> None:
        check(lib().srg_scene_set_form(self.handle, form, tile_cfg))

    def tile_shears(self) -> list:
        """Tile shear (lines per 32 columns) in use for each burst."""
        out = []
        for i in range(len(self.bursts)):
            v = C.c_int()
            check(lib().srg_scene_tile_shear(self.handle, i, C.byref(v)))
            out.append(int(v.value))
        return out

    def shape(self) -> int:
        return int(lib().srg_scene_shape(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().srg_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
