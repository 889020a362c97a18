"""ctypes bindings to the oracle -- TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the reference's per-burst backprojection:

* ``Oracle``    this project's C restatement (oracle/liboracle.so);
* ``RefCPU``    the reference's own sentinel/azimuth_compress_cpu.c compiled
                unmodified (oracle/_ref/libref_cpu.so, built by `make ref`
                where the reference tree is mounted).

Only the tests, the smoke check and the benchmark's CPU-baseline leg use
this module, always as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_cpu.so")

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_sp = C.POINTER(C.c_int16)


def build(ref: bool = False) -> None:
    """Compile the oracle (and, if asked and possible, the reference)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, t):
    return a.ctypes.data_as(t)


class Opts(C.Structure):
    _fields_ = [("gpu_lerp", C.c_int), ("gpu_scale", C.c_int), ("nthreads", C.c_int)]


class Oracle:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.srg_oracle_pixelint.restype = C.c_int64
        L.srg_oracle_burst.restype = C.c_int64
        L.srg_oracle_count_terms.restype = C.c_int64

    # -- building blocks ------------------------------------------------
    def limits(self, b):
        fl, ll, fp, lp = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ll4 = _d(b.latlons)
        self.lib.srg_oracle_limits(_ptr(ll4, _dp), C.c_double(b.firstlat), C.c_double(b.deltalat),
                                   C.c_double(b.firstlon), C.c_double(b.deltalon),
                                   C.c_int(b.demwidth), C.c_int(b.demlength), C.byref(fl),
                                   C.byref(ll), C.byref(fp), C.byref(lp))
        return fl.value, ll.value, fp.value, lp.value

    def setxyz(self, b, firstline, nlines, firstpix, lastpix):
        W = b.demwidth
        slab = np.ascontiguousarray(b.dem[firstline:firstline + nlines], np.int16)
        xyz = np.zeros((nlines, W, 3))
        fit = np.zeros((nlines, 9))
        self.lib.srg_oracle_setxyz(_ptr(slab, _sp), _ptr(xyz, _dp), _ptr(fit, _dp), C.c_int(W),
                                   C.c_double(b.firstlat), C.c_double(b.deltalat),
                                   C.c_double(b.firstlon), C.c_double(b.deltalon),
                                   C.c_int(firstline), C.c_int(nlines), C.c_int(firstpix),
                                   C.c_int(lastpix))
        return xyz, fit

    def line_coefs(self, b, xyzfit):
        nl = xyzfit.shape[0]
        coef = np.zeros((nl, 3))
        xyzfit = _d(xyzfit)
        to, xx, vv = _d(b.timeorbit), _d(b.xx), _d(b.vv)
        xm, vm = _d(b.xyz_mid), _d(b.vel_mid)
        self.lib.srg_oracle_line_coefs(_ptr(xyzfit, _dp), C.c_int(nl), _ptr(to, _dp),
                                       _ptr(xx, _dp), _ptr(vv, _dp), C.c_int(len(to)),
                                       C.c_double(b.tmid), _ptr(xm, _dp), _ptr(vm, _dp),
                                       C.c_double(b.wvl), C.c_double(b.angc0),
                                       C.c_double(b.angc1), C.c_double(b.prf),
                                       C.c_int(b.rawdatalines), _ptr(coef, _dp))
        return coef

    def setazoff(self, b, coef, firstpix, lastpix):
        nl = coef.shape[0]
        az = np.zeros((nl, b.demwidth))
        coef = _d(coef)
        self.lib.srg_oracle_setazoff(_ptr(coef, _dp), _ptr(az, _dp), C.c_int(b.demwidth),
                                     C.c_int(nl), C.c_int(firstpix), C.c_int(lastpix),
                                     C.c_int(b.aperture), C.c_int(b.rawdatalines))
        return az

    def pixelint(self, b, xyz, azoff, gpu_lerp=1, gpu_scale=1, nthreads=0, want_acc=False):
        nl, W = azoff.shape
        out = np.zeros((nl, W), np.complex64)
        acc = np.zeros((nl, W), np.complex128) if want_acc else None
        burst = np.ascontiguousarray(b.burst, np.complex64)
        sat = _d(b.satloc)
        xyz = _d(xyz)
        azoff = _d(azoff)
        o = Opts(gpu_lerp, gpu_scale, nthreads)
        terms = self.lib.srg_oracle_pixelint(
            burst.ctypes.data_as(_fp), _ptr(sat, _dp), _ptr(xyz, _dp), _ptr(azoff, _dp),
            C.c_int(W), C.c_int(b.aperture), C.c_int(b.rawdatalines), C.c_int(b.samples),
            C.c_double(b.rngstart), C.c_double(b.rngend), C.c_double(b.dmrg), C.c_double(b.wvl),
            C.c_int(nl), out.ctypes.data_as(_fp),
            acc.ctypes.data_as(_dp) if acc is not None else None, C.byref(o))
        return out, acc, int(terms)

    def pulse_orbit(self, times, b):
        """Per-pulse positions and velocities ([P][3] each) by the window rule
        of sentinel/sentineltimingsub.f90:55-63 (unclamped); raises if a pulse
        time falls where the reference would read outside the vectors."""
        t = _d(times)
        P = t.shape[0]
        pos, vel = np.zeros((P, 3)), np.zeros((P, 3))
        to, xx, vv = _d(b.timeorbit), _d(b.xx), _d(b.vv)
        bad = self.lib.srg_oracle_pulse_orbit(_ptr(t, _dp), C.c_int(P), _ptr(to, _dp),
                                              _ptr(xx, _dp), _ptr(vv, _dp), C.c_int(len(to)),
                                              _ptr(pos, _dp), _ptr(vel, _dp))
        if bad:
            raise ValueError(f"{bad} pulse times outside the state-vector window")
        return pos, vel

    def count_terms(self, b, nthreads=0):
        """Executed-term count of one burst (limits, ECEF, azimuth centres,
        azoff, then pixelint's window and range test without the sum)."""
        fl, ll, fp, lp = self.limits(b)
        nl = ll - fl + 1
        xyz, fit = self.setxyz(b, fl, nl, fp, lp)
        az = self.setazoff(b, self.line_coefs(b, fit), fp, lp)
        return int(self.lib.srg_oracle_count_terms(
            _ptr(_d(b.satloc), _dp), _ptr(xyz, _dp), _ptr(az, _dp), C.c_int(b.demwidth),
            C.c_int(b.aperture), C.c_int(b.rawdatalines), C.c_double(b.rngstart),
            C.c_double(b.rngend), C.c_double(b.dmrg), C.c_int(nl), C.c_int(nthreads)))

    # -- one burst --------------------------------------------------------
    def stages(self, b, gpu_lerp=1, gpu_scale=1, nthreads=0, want_acc=False):
        """Every intermediate of one burst: dict(firstline, nlines, firstpix,
        lastpix, xyz, xyzfit, coef, azoff, out, acc, terms)."""
        fl, ll, fp, lp = self.limits(b)
        nl = ll - fl + 1
        xyz, fit = self.setxyz(b, fl, nl, fp, lp)
        coef = self.line_coefs(b, fit)
        az = self.setazoff(b, coef, fp, lp)
        out, acc, terms = self.pixelint(b, xyz, az, gpu_lerp, gpu_scale, nthreads, want_acc)
        return dict(firstline=fl, nlines=nl, firstpix=fp, lastpix=lp, xyz=xyz, xyzfit=fit,
                    coef=coef, azoff=az, out=out, acc=acc, terms=terms)

    def burst_geo(self, b, geo=None, gpu=True, nthreads=0):
        """Merge one burst into a [L][W] complex64 raster (GPU or CPU rule)."""
        if geo is None:
            geo = np.zeros((b.demlength, b.demwidth), np.complex64)
        burst = np.ascontiguousarray(b.burst, np.complex64)
        dem = np.ascontiguousarray(b.dem, np.int16)
        o = Opts(1 if gpu else 0, 1 if gpu else 0, nthreads)
        fl, nl = C.c_int(), C.c_int()
        args = self._common(b)
        terms = self.lib.srg_oracle_burst(
            burst.ctypes.data_as(_fp), args["satloc"], C.c_int(b.rawdatalines),
            C.c_int(b.samples), C.c_int(b.demwidth), C.c_int(b.demlength), _ptr(dem, _sp),
            geo.ctypes.data_as(_fp), C.c_double(b.deltalat), C.c_double(b.deltalon),
            C.c_double(b.firstlat), C.c_double(b.firstlon), args["latlons"], args["timeorbit"],
            args["xx"], args["vv"], C.c_int(b.numstatevec), C.c_double(b.rngstart),
            C.c_double(b.rngend), C.c_double(b.tmid), args["xyz_mid"], args["vel_mid"],
            C.c_double(b.dmrg), C.c_double(b.wvl), C.c_int(b.aperture), C.c_double(b.angc0),
            C.c_double(b.angc1), C.c_double(b.prf), None, C.byref(fl), C.byref(nl), C.byref(o))
        return geo, int(terms)

    def _common(self, b):
        keep = {k: _d(getattr(b, k)) for k in
                ("satloc", "latlons", "timeorbit", "xx", "vv", "xyz_mid", "vel_mid")}
        self._keep = keep
        return {k: _ptr(v, _dp) for k, v in keep.items()}


def call_33(fn, b, fdout: int, fddem: int, burst=None):
    """Call a 33-argument by-reference entry (reference layout) for burst b."""
    burst = np.ascontiguousarray(b.burst if burst is None else burst, np.complex64)
    dd = {k: _d(getattr(b, k)) for k in
          ("satloc", "latlons", "timeorbit", "xx", "vv", "xyz_mid", "vel_mid", "pulse_time")}
    ints = {k: C.c_int(v) for k, v in dict(
        P=b.rawdatalines, S=b.samples, W=b.demwidth, L=b.demlength, fo=fdout, fd=fddem,
        n=b.numstatevec, ap=b.aperture, iap=b.iaperture).items()}
    dbl = {k: C.c_double(getattr(b, k)) for k in
           ("deltalat", "deltalon", "firstlat", "firstlon", "rngstart", "rngend", "tstart",
            "tend", "tmid", "dtaz", "dmrg", "wvl", "angc0", "angc1", "prf")}
    r = C.byref
    fn(burst.ctypes.data_as(_fp), _ptr(dd["satloc"], _dp), r(ints["P"]), r(ints["S"]),
       r(ints["W"]), r(ints["L"]), r(ints["fo"]), r(ints["fd"]), r(dbl["deltalat"]),
       r(dbl["deltalon"]), r(dbl["firstlat"]), r(dbl["firstlon"]), _ptr(dd["latlons"], _dp),
       _ptr(dd["timeorbit"], _dp), _ptr(dd["xx"], _dp), _ptr(dd["vv"], _dp), r(ints["n"]),
       r(dbl["rngstart"]), r(dbl["rngend"]), r(dbl["tstart"]), r(dbl["tend"]), r(dbl["tmid"]),
       _ptr(dd["xyz_mid"], _dp), _ptr(dd["vel_mid"], _dp), _ptr(dd["pulse_time"], _dp),
       r(dbl["dtaz"]), r(dbl["dmrg"]), r(dbl["wvl"]), r(ints["ap"]), r(ints["iap"]),
       r(dbl["angc0"]), r(dbl["angc1"]), r(dbl["prf"]))


def run_33_files(fn, b, geo_init=None, timing=None, tmpdir=None, read_back=True):
    """Run a 33-arg entry with a temporary DEM file and .geo file; return the
    resulting [L][W] complex64 raster (None without read_back).  timing
    (dict, optional) receives the wall time of the entry call alone as
    timing["call_s"]; tmpdir: where the files go (default: the temp dir)."""
    with tempfile.TemporaryDirectory(dir=tmpdir) as td:
        dem_path = os.path.join(td, "elevation.dem")
        geo_path = os.path.join(td, "scene.geo")
        np.ascontiguousarray(b.dem, np.int16).tofile(dem_path)
        if geo_init is None:
            with open(geo_path, "wb") as f:   # a zero-filled raster
                f.truncate(b.demlength * b.demwidth * 8)
        else:
            np.ascontiguousarray(geo_init, np.complex64).tofile(geo_path)
        fddem = os.open(dem_path, os.O_RDWR)
        fdout = os.open(geo_path, os.O_RDWR)
        try:
            import time as _t
            t0 = _t.perf_counter()
            call_33(fn, b, fdout, fddem)
            if timing is not None:
                timing["call_s"] = _t.perf_counter() - t0
            # The reference leaves its fdopen() stream unflushed; write out its
            # buffered tail before the descriptor is closed.
            C.CDLL(None).fflush(None)
        finally:
            os.close(fddem)
            os.close(fdout)
        if not read_back:
            return None
        return np.fromfile(geo_path, np.complex64).reshape(b.demlength, b.demwidth)


class RefCPU:
    """The reference CPU backprojection, compiled from the reference sources."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)

    def pixelint(self, b, xyz, azoff, out=None):
        nl, W = azoff.shape
        out = np.zeros((nl, W), np.complex64) if out is None else out
        burst = np.ascontiguousarray(b.burst, np.complex64)
        sat, xyz, azoff = _d(b.satloc), _d(xyz), _d(azoff)
        self.lib.pixelint(burst.ctypes.data_as(_fp), _ptr(sat, _dp), _ptr(xyz, _dp),
                          _ptr(azoff, _dp), C.c_int(W), C.c_int(b.aperture),
                          C.c_int(b.iaperture), C.c_int(b.rawdatalines), C.c_int(b.samples),
                          C.c_double(b.rngstart), C.c_double(b.rngend), C.c_double(b.dmrg),
                          C.c_double(b.wvl), out.ctypes.data_as(_fp), C.c_int(nl))
        return out

    def setxyz(self, b, firstline, nlines, firstpix, lastpix):
        W = b.demwidth
        slab = np.ascontiguousarray(b.dem[firstline:firstline + nlines], np.int16)
        xyz = np.zeros((nlines, W, 3))
        fit = np.zeros((nlines, 9))
        az = np.zeros((nlines, W))
        self.lib.setxyz(_ptr(slab, _sp), _ptr(xyz, _dp), _ptr(fit, _dp), _ptr(az, _dp),
                        C.c_int(W), C.c_double(b.firstlat), C.c_double(b.deltalat),
                        C.c_double(b.firstlon), C.c_double(b.deltalon), C.c_int(firstline),
                        C.c_int(nlines), C.c_int(firstpix), C.c_int(lastpix))
        return xyz, fit

    def setazoff(self, b, coef, firstpix, lastpix, fill=-1.0):
        nl = coef.shape[0]
        az = np.full((nl, b.demwidth), fill)
        coef = _d(coef)
        self.lib.setazoff(_ptr(coef, _dp), _ptr(az, _dp), C.c_int(b.demwidth), C.c_int(nl),
                          C.c_int(firstpix), C.c_int(lastpix), C.c_int(b.aperture),
                          C.c_int(b.rawdatalines))
        return az

    def azimuth_compress_cpu(self, b, geo_init=None, timing=None):
        return run_33_files(self.lib.azimuth_compress_cpu_, b, geo_init, timing)
