"""CPU restatement of the reference's interferogram program (test infrastructure).

Follows int/crossmul.f90 step for step, per output line (the reference's
OpenMP loop body, crossmul.f90:95-185):

* lines (line-1)*looksdn+1 .. line*looksdn of both files (:103-108; the same
  data for both when the two names are equal);
* masks from the unscaled input: per look window the complex sum over the
  looksdn lines (sum(in, 2)) and then over looksac samples; |.| <= 1e-6 marks
  the window empty (:110-125);
* in * scale (:127-128);
* upsampling by 2 across: nnn = first 2^i >= na (i = 1..24, :69-73); forward
  DFT of the zero-padded line (FFTW sign -1, unnormalised), bins [0, nnn/2) to
  [0, nnn/2) and [nnn/2, nnn) to [2nnn - nnn/2, 2nnn) of a zeroed 2nnn array,
  inverse DFT (sign +1, unnormalised), / nnn / 2 (:130-153);
* igram = up1 * conj(up2), amp = (|up1|^2, |up2|^2) (:155-156); samples 2j-1
  and 2j summed into j (:158-161); summed over the looksdn lines (:164-165);
  summed over looksac samples (:168-172); amp -> (sqrt re, sqrt im) (:173);
  masked windows set to 0 (:176-184).

FFTW 3.3.9 (single precision, ``sfftw_*``) is not vendored in the reference
and not installed here; its published transform is the plain DFT with the
stated signs, which numpy.fft computes (``fft`` = sign -1; ``ifft`` * N =
sign +1, unnormalised).  Computed in complex128 by default: the reference's
own single-precision rounding is not reproduced, so parity with it is at the
level of FP32 rounding and this restatement is unpinned by golden vectors
(the reference ships none).
"""
from __future__ import annotations

import numpy as np


def fft_length(na: int) -> int:
    """crossmul.f90:69-73: the first 2**i >= na, i = 1..24."""
    for i in range(1, 25):
        if 2 ** i >= na:
            return 2 ** i
    return 2 ** 24


def upsample2(lines: np.ndarray, nnn: int, dtype=np.complex128) -> np.ndarray:
    """[n, na] -> [n, 2*nnn] (crossmul.f90:130-153)."""
    n, na = lines.shape
    buf = np.zeros((n, nnn), dtype)
    buf[:, :na] = lines
    X = np.fft.fft(buf, axis=1)
    up = np.zeros((n, 2 * nnn), dtype)
    up[:, :nnn // 2] = X[:, :nnn // 2]
    up[:, 2 * nnn - nnn // 2:] = X[:, nnn // 2:]
    t = np.fft.ifft(up, axis=1) * (2 * nnn)  # unnormalised inverse (sign +1)
    return (t / nnn / 2.0).astype(dtype)


def crossmul(in1: np.ndarray, in2: np.ndarray, looksac: int = 1, looksdn: int | None = None,
             scale: float = 1.0, mask: bool = True, nvalid: int | None = None,
             dtype=np.complex128):
    """Interferogram and amplitude images of two [nd][na] complex images.

    Returns (igram, amp), each [nvalid // looksdn][na // looksac]."""
    in1 = np.asarray(in1)
    in2 = np.asarray(in2)
    nd, na = in1.shape
    if looksdn is None:
        looksdn = looksac
    if nvalid is None:
        nvalid = nd
    nnn = fft_length(na)
    nout, ncol = nvalid // looksdn, na // looksac
    igram_out = np.zeros((nout, ncol), np.complex64)
    amp_out = np.zeros((nout, ncol), np.complex64)
    for line in range(nout):
        a = in1[line * looksdn:(line + 1) * looksdn].astype(dtype)
        b = in2[line * looksdn:(line + 1) * looksdn].astype(dtype)
        keep = np.ones(ncol, bool)
        if mask:
            for x in (a, b):
                s = x.sum(axis=0)[:ncol * looksac].reshape(ncol, looksac).sum(axis=1)
                keep &= ~(np.abs(s) <= 1e-6)
        u1 = upsample2(a * scale, nnn, dtype)
        u2 = upsample2(b * scale, nnn, dtype)
        ig = u1[:, :2 * na] * np.conj(u2[:, :2 * na])
        am = (np.abs(u1[:, :2 * na]) ** 2) + 1j * (np.abs(u2[:, :2 * na]) ** 2)
        ig = ig[:, 0::2] + ig[:, 1::2]                     # reclaim the two across
        am = am[:, 0::2] + am[:, 1::2]
        igacc = ig.sum(axis=0)                             # looks down
        amacc = am.sum(axis=0)
        igt = igacc[:ncol * looksac].reshape(ncol, looksac).sum(axis=1)  # looks across
        amt = amacc[:ncol * looksac].reshape(ncol, looksac).sum(axis=1)
        amt = np.sqrt(amt.real) + 1j * np.sqrt(amt.imag)
        igt[~keep] = 0
        amt[~keep] = 0
        igram_out[line] = igt
        amp_out[line] = amt
    return igram_out, amp_out
