"""Range compression (sentinel/processsub.f90:86-123): the library's host
replica and the oracle's restatement against each other and a point-target
identity on the CPU; the CUDA path (srg_range_compress_device through the C
ABI) against the oracle on the GPU."""
import numpy as np
import pytest

import rangecomp as orc  # oracle/rangecomp.py

# IW-like pulse: 3/7 * 4 * fref MHz sampling, ~52 us pulse, ~0.78 MHz/us ramp
FS = float(np.float32(3.0 / 7.0 * 4.0 * 37.53472224))
PULSE = dict(samplefreq=FS, startfreq=-20.2, ramprate=0.7792, pulselength=52.4)


def test_library_replica_matches_restatement():
    from srg_b200 import api
    rep, npts = api.range_replica(**PULSE)
    want, wnpts = orc.replica(**PULSE)
    assert npts == wnpts == int(np.float32(PULSE["pulselength"]) * np.float32(FS))
    assert np.array_equal(rep, want)


def test_overlap_save_gives_the_kept_samples():
    """The identity the fused GPU kernel rests on, checked on the restatement:
    the kept samples of the 32,768-point circular correlation are a linear
    correlation (the wrap never reaches n < nvalid), so overlap-save with
    8,192-point segments of 8,192 - npts + 1 outputs, filter
    4 conj(DFT_8192(replica)) and the inverse as the conjugate of a forward
    transform of the conjugate, gives them to FP64 rounding; over segment
    boundaries and a line's last samples too."""
    M = 8192
    rep, npts = orc.replica(**PULSE)
    rng = np.random.default_rng(11)
    for nsamps in (9000, 21000, 32768):
        x = (rng.standard_normal((2, nsamps)) + 1j * rng.standard_normal((2, nsamps))).astype(np.complex64)
        want = orc.range_compress(x, **PULSE)
        nvalid, L = nsamps - npts, M - npts + 1
        H = (orc.RANFFT / M) * np.conj(np.fft.fft(np.concatenate(
            [rep[:npts].astype(np.complex128), np.zeros(M - npts)])))
        got = np.zeros((2, nvalid), np.complex128)
        for s0 in range(0, nvalid, L):
            seg = np.zeros((2, M), np.complex128)
            n = min(M, nsamps - s0)
            seg[:, :n] = x[:, s0:s0 + n]
            y = np.conj(np.fft.fft(np.conj(np.fft.fft(seg, axis=1) * H), axis=1))
            m = min(L, nvalid - s0)
            got[:, s0:s0 + m] = y[:, :m]
        rms = np.sqrt(np.mean(np.abs(want) ** 2))
        assert np.abs(got - want).max() / rms < 1e-6


def test_point_target_compresses_to_a_peak_of_ranfft():
    # correlation with the replica (sum |chirp|^2 / npts = 1), times 32,768 from
    # the unnormalised inverse transform
    rep, npts = orc.replica(**PULSE)
    chirp = rep[:npts] * npts                       # unit-amplitude pulse
    nsamps, d = 12000, 4321
    line = np.zeros((1, nsamps), np.complex64)
    line[0, d:d + npts] = chirp
    out = orc.range_compress(line, **PULSE)
    assert out.shape == (1, nsamps - npts)
    k = int(np.argmax(np.abs(out[0])))
    assert k == d
    assert abs(out[0, k] / orc.RANFFT - 1.0) < 1e-5


gpu = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def _lines(rng, nlines, nsamps, ntargets=5, pulse=PULSE):
    x = (rng.standard_normal((nlines, nsamps)) + 1j * rng.standard_normal((nlines, nsamps))).astype(np.complex64)
    rep, npts = orc.replica(**pulse)
    for l in range(nlines):
        for d in rng.integers(0, nsamps - npts, ntargets):
            x[l, d:d + npts] += 10.0 * rep[:npts] * npts
    return x


@gpu
@pytest.mark.parametrize("nlines,nsamps,pad_in,pad_out", [(300, 20000, 0, 0), (7, 9000, 13, 5),
                                                          (1, 32768, 0, 0)])
def test_gpu_range_compress_matches_oracle(torch_cuda, nlines, nsamps, pad_in, pad_out):
    torch = torch_cuda
    from srg_b200 import api
    rng = np.random.default_rng(nlines + nsamps)
    x = _lines(rng, nlines, nsamps)
    want = orc.range_compress(x, **PULSE)
    tin = torch.zeros((nlines, nsamps + pad_in), dtype=torch.complex64, device="cuda")
    tin[:, :nsamps] = torch.from_numpy(x).cuda()
    nvalid = want.shape[1]
    tout = torch.zeros((nlines, nvalid + pad_out), dtype=torch.complex64, device="cuda")
    api.range_compress(tin, nsamps=nsamps, out=tout[:, :nvalid], **PULSE)
    got = tout[:, :nvalid].cpu().numpy()
    rms = np.sqrt(np.mean(np.abs(want) ** 2))
    err = np.abs(got.astype(np.complex128) - want).max() / rms
    assert err < 2e-5, err
    if pad_out:
        assert torch.count_nonzero(tout[:, nvalid:]).item() == 0


@gpu
@pytest.mark.parametrize("pulselength", [PULSE["pulselength"], 80.0])
def test_gpu_range_compress_both_paths(torch_cuda, pulselength):
    """Pulses of up to 4,096 samples take the fused overlap-save kernel (8,192-
    point segments), longer ones the cuFFT path (32,768-point rows); both
    match the oracle at every kept sample, lines with targets near both ends
    included (the lines of the test above, plus one target per line at an
    edge or a segment boundary)."""
    torch = torch_cuda
    from srg_b200 import api
    pulse = dict(PULSE, pulselength=pulselength)
    rep, npts = orc.replica(**pulse)
    assert (npts <= 4096) == (pulselength == PULSE["pulselength"])
    rng = np.random.default_rng(npts)
    nlines, nsamps = 9, 21000
    x = _lines(rng, nlines, nsamps, pulse=pulse)
    for l, d in enumerate([0, 1, nsamps - npts, nsamps - npts - 1, 4821, 4822, 9000, 13000, 17000]):
        d = min(d, nsamps - npts)
        x[l, d:d + npts] += 10.0 * rep[:npts] * npts
    want = orc.range_compress(x, **pulse)
    tin = torch.from_numpy(x).cuda()
    tout = torch.zeros((nlines, want.shape[1]), dtype=torch.complex64, device="cuda")
    api.range_compress(tin, nsamps=nsamps, out=tout, **pulse)
    got = tout.cpu().numpy()
    err = np.abs(got.astype(np.complex128) - want).max() / np.sqrt(np.mean(np.abs(want) ** 2))
    assert err < 2e-5, err


@gpu
def test_gpu_range_compress_rejects_long_lines(torch_cuda):
    torch = torch_cuda
    from srg_b200 import _lib, api
    x = torch.zeros((2, 32769), dtype=torch.complex64, device="cuda")
    with pytest.raises(_lib.SrgError):
        api.range_compress(x, **PULSE)
