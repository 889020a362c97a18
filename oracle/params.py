"""Per-burst scalars of the azimuth_compress_ call -- TEST INFRASTRUCTURE ONLY.

Restatement (numpy scalars, so every step rounds in the precision the
Fortran uses) of what sentinel/backprojectgpusub.f90 derives before each
call: burstparams (:406-429), fdopcoefs (:262-309) with linfit (:381-403),
the aperture (:190-209) and the azimuth / range limits (:213-227); with the
header field readers and samplefrequency of sentinel/processsub.f90:163-211.

gfortran is not installed, so the Fortran cannot be run here; the precision
of every step is read off the source: literals without a d exponent are
default REAL (single precision), so fref in fdopcoefs, the 1.e6 / 1.e-6
factors and the wavelength are single-precision values promoted to double;
ang, prf and t in fdopcoefs are REAL arrays; linfit accumulates REAL
products in REAL*8 and returns REAL coefficients; angc0 and angc1 are
implicitly REAL inside fdopcoefs.  Only the tests use this module, as the
checker of srg_burst_params.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32
f64 = np.float64

FREF_D = f64(37.53472224)          # burstparams, samplefrequency: 37.53472224d0
FREF_S = f64(f32(37.53472224))     # fdopcoefs: fref=37.53472224 (REAL literal)
SOL = f64(299792458.0)

# processsub.f90:176-211 -- (numerator, denominator) of each decimation code
_FRACTIONS = {0: (3, 4), 1: (2, 3), 3: (5, 9), 4: (4, 9), 5: (3, 8), 6: (1, 3), 7: (1, 6),
              8: (3, 7), 9: (5, 16), 10: (3, 26), 11: (4, 11)}


def in2(b, o):
    """processsub.f90:163-167, 1-based byte o+1 -> 0-based offset o."""
    return int(b[o + 1]) + 256 * int(b[o])


def in3(b, o):
    return int(b[o + 2]) + 256 * int(b[o + 1]) + 65536 * int(b[o])


def d8(b, o):
    return f64(np.frombuffer(bytes(b[o:o + 8]), dtype="<f8")[0])


def samplefrequency(code):
    n, d = _FRACTIONS[code]
    return f64(f32(f32(n) / f32(d)) * f32(4.0)) * FREF_D


def burst_params(headers: np.ndarray, satvel: np.ndarray, samples: int) -> dict:
    """headers: [P][80] uint8 (each line's first 10 complex64 samples, as
    bytes); satvel [P][3]; samples = rangesamples incl. the 10 header words."""
    P = headers.shape[0]
    h0 = headers[0]
    # burstparams (:406-429)
    starttime = d8(h0, 68)
    prf = FREF_D / f64(in3(h0, 50)) * f64(f32(1.e6))
    samplefreq = samplefrequency(int(h0[40]) & 255) * f64(f32(1.e6))
    swst = f64(in3(h0, 53)) / FREF_D * f64(f32(1.e-6))
    irank = int(h0[49]) & 31
    pri = f64(in3(h0, 50)) / FREF_D * f64(f32(1.e-6))
    range0 = SOL / f64(2.0) * (f64(irank) * pri + swst) + f64(60.0)
    wvl = f64(f32(0.05546576))
    # fdopcoefs (:262-309)
    ang = np.empty(P, f32)
    t = np.empty(P, f32)
    half = f32(P) / f32(2.0)
    for i in range(1, P + 1):
        h = headers[i - 1]
        word = in2(h, 60)
        azimuthbeam = word & 1023
        ang[i - 1] = f32(f32(f32(azimuthbeam) / f32(1024.0)) * f32(1.8)) - f32(0.9)
        prf_i = f32(FREF_S / f64(in3(h, 50)) * f64(f32(1.e6)))
        t[i - 1] = f32(f32(i) - half) / prf_i
    x, y = t[20:P - 20], ang[20:P - 20]
    npts = P - 40
    sumx = sumx2 = sumxy = sumy = f64(0.0)
    for xi, yi in zip(x, y):
        sumx = sumx + f64(xi)
        sumx2 = sumx2 + f64(f32(xi * xi))
        sumxy = sumxy + f64(f32(xi * yi))
        sumy = sumy + f64(yi)
    den = f64(npts) * sumx2 - sumx * sumx
    angc1 = f64(f32((f64(npts) * sumxy - sumx * sumy) / den))
    angc0 = f64(f32((sumy * sumx2 - sumx * sumxy) / den))
    # aperture (:190-209)
    re, ht = f64(6378137.0), f64(700000.0)
    pi = f64(4.0) * f64(math.atan2(1.0, 1.0))
    v = np.asarray(satvel[P // 2 - 1], f64)
    vmag = f64(math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])) * (re / (re + ht))
    aperturetime = (range0 * wvl / f64(2) / vmag / vmag * prf) / \
        (f64(1.0) + range0 * angc1 * pi / f64(180.0) / vmag)
    aperture = int(aperturetime * prf * f64(0.5))
    # limits (:213-227)
    tstart = starttime
    dtaz = f64(1.0) / prf
    tend = tstart + f64(P - 1) * dtaz
    tmid = f64(0.5) * (tstart + tend)
    rngstart = (f64(2) * range0 / SOL) * SOL / f64(2.0)
    dmrg = SOL / f64(2.0) / samplefreq
    rngend = rngstart + f64(samples - 1) * dmrg
    return dict(starttime=starttime, prf=prf, samplefreq=samplefreq, pri=pri, range0=range0,
                wvl=wvl, angc0=angc0, angc1=angc1, tstart=tstart, tend=tend, tmid=tmid,
                dtaz=dtaz, rngstart=rngstart, rngend=rngend, dmrg=dmrg, aperture=aperture)
