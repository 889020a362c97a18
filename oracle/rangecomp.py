"""CPU restatement of the reference's range compression (test infrastructure).

Follows sentinel/processsub.f90:86-123:

* pulse samples npts = int(pulselength * samplefreq), a product of two
  real*4 values (:94), and nvalid = nsamps - npts (:95);
* the replica (:101-107): for j = 1..npts, t = (j-1)/samplefreq evaluated in
  real*4, phase = 2 pi startfreq t + pi ramprate t^2 in real*8, the sample
  cmplx(cos, sin) rounded to complex*8 and divided by npts; zero elsewhere;
  its 32,768-point forward DFT (FFTW sign -1, unnormalised) (:108);
* per line (:111-119): the samples zero-padded to 32,768, forward DFT, times
  the conjugate replica spectrum, inverse DFT (sign +1, unnormalised), the
  first nvalid samples kept (:122).

FFTW 3.3.9 is not vendored in the reference and not installed here; its
published transforms are the plain DFTs with these signs, which numpy.fft
computes (``fft``; ``ifft`` * N).  The transforms run in complex128: parity
with the reference's single-precision FFTW is at FP32 rounding and unpinned
by golden vectors (the reference ships none).
"""
from __future__ import annotations

import numpy as np

RANFFT = 32768  # processsub.f90:38


def replica(samplefreq: float, startfreq: float, ramprate: float, pulselength: float,
            n: int = RANFFT):
    """(complex64 [n] zero-padded replica, npts)."""
    sf = np.float32(samplefreq)
    npts = int(np.float32(pulselength) * sf)
    j = np.arange(npts, dtype=np.float32)
    t = (j / sf).astype(np.float64)
    phase = 2.0 * np.pi * np.float64(np.float32(startfreq)) * t + np.pi * np.float64(np.float32(ramprate)) * t * t
    rep = np.zeros(n, np.complex64)
    c = np.cos(phase).astype(np.float32) / np.float32(npts)
    s = np.sin(phase).astype(np.float32) / np.float32(npts)
    rep[:npts] = c + 1j * s
    return rep, npts


def range_compress(lines: np.ndarray, samplefreq: float, startfreq: float, ramprate: float,
                   pulselength: float, nsamps: int | None = None) -> np.ndarray:
    """[nlines][>= nsamps] complex -> [nlines][nvalid] complex64."""
    lines = np.asarray(lines)
    nsamps = lines.shape[1] if nsamps is None else nsamps
    rep, npts = replica(samplefreq, startfreq, ramprate, pulselength)
    nvalid = nsamps - npts
    ref = np.fft.fft(rep.astype(np.complex128))
    buf = np.zeros((lines.shape[0], RANFFT), np.complex128)
    buf[:, :nsamps] = lines[:, :nsamps]
    spec = np.fft.fft(buf, axis=1) * np.conj(ref)[None, :]
    out = np.fft.ifft(spec, axis=1) * RANFFT
    return out[:, :nvalid].astype(np.complex64)
