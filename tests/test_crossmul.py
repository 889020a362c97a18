"""Interferogram formation (int/crossmul.f90): the oracle's restatement
against the algorithm's own identities on the CPU, and the CUDA path
(srg_crossmul_device / srg_crossmul_stack_device through the C ABI) against
the oracle on the GPU."""
import os
import tempfile

import numpy as np
import pytest

import crossmul as ox  # oracle/crossmul.py


def _img(rng, nd, na, amp=1.0):
    return ((rng.standard_normal((nd, na)) + 1j * rng.standard_normal((nd, na))) * amp).astype(np.complex64)


# ---------------------------------------------------------------- CPU (oracle)

def test_fft_length():
    assert [ox.fft_length(n) for n in (1, 2, 3, 5, 2400, 4096, 4097)] == [2, 2, 4, 8, 4096, 4096, 8192]


def test_upsample_even_samples_are_half_the_input():
    # zero-padding the spectrum keeps the original samples (halved by the
    # reference's / nnn / 2) at the even positions
    x = _img(np.random.default_rng(1), 3, 37)
    up = ox.upsample2(x.astype(np.complex128), ox.fft_length(37))
    np.testing.assert_allclose(up[:, 0:74:2], x / 2.0, atol=1e-6)


def test_upsample_from_odd_samples():
    """The identity the fused GPU kernels rest on, on the restatement: with
    the spectrum X spread as the reference spreads it, the unnormalised
    2nnn-point inverse u has u[2n] = nnn x[n] and u[2n + 1] = the nnn-point
    inverse of X[k] s_k exp(i pi k / nnn), s_k = -1 for the bins moved to
    the top (upsample2 returns u / nnn / 2)."""
    rng = np.random.default_rng(12)
    for na in (2049, 2600, 4096):
        x = _img(rng, 2, na).astype(np.complex128)
        nnn = ox.fft_length(na)
        up = ox.upsample2(x, nnn) * nnn * 2.0
        xp = np.zeros((2, nnn), np.complex128)
        xp[:, :na] = x
        k = np.arange(nnn)
        tw = np.where(k < nnn // 2, 1.0, -1.0) * np.exp(1j * np.pi * k / nnn)
        odd = np.fft.ifft(np.fft.fft(xp, axis=1) * tw, axis=1) * nnn
        scale = np.abs(up).max()
        assert np.abs(up[:, 0::2] - nnn * xp).max() / scale < 1e-12
        assert np.abs(up[:, 1::2] - odd).max() / scale < 1e-12


def test_identical_images_give_real_power():
    x = _img(np.random.default_rng(2), 12, 50)
    ig, am = ox.crossmul(x, x, looksac=2, looksdn=3, mask=False)
    assert np.abs(ig.imag).max() <= 1e-6 * np.abs(ig.real).max()
    np.testing.assert_allclose(ig.real, am.real ** 2, rtol=1e-5)
    np.testing.assert_allclose(am.real, am.imag, rtol=1e-6)


def test_constant_phase_offset_is_recovered():
    x = _img(np.random.default_rng(3), 8, 64)
    phi = 0.7
    y = (x * np.exp(-1j * phi)).astype(np.complex64)
    ig, _ = ox.crossmul(x, y, looksac=4, looksdn=2, mask=False)
    np.testing.assert_allclose(np.angle(ig), phi, atol=1e-5)


def test_looks_are_sums_of_single_look_samples():
    rng = np.random.default_rng(4)
    x, y = _img(rng, 12, 30), _img(rng, 12, 30)
    one, _ = ox.crossmul(x, y, looksac=1, looksdn=1, mask=False)
    ml, _ = ox.crossmul(x, y, looksac=3, looksdn=4, mask=False)
    want = one[:12].reshape(3, 4, 10, 3).sum(axis=(1, 3))
    np.testing.assert_allclose(ml, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


def test_mask_zeroes_empty_windows_only():
    rng = np.random.default_rng(5)
    x, y = _img(rng, 8, 40), _img(rng, 8, 40)
    x[:, 10:20] = 0
    ig, am = ox.crossmul(x, y, looksac=2, looksdn=2, mask=True)
    assert np.all(ig[:, 5:10] == 0) and np.all(am[:, 5:10] == 0)
    assert np.all(np.abs(ig[:, :5]) > 0) and np.all(np.abs(ig[:, 10:]) > 0)
    ig2, _ = ox.crossmul(x, y, looksac=2, looksdn=2, mask=False)
    assert np.all(np.abs(ig2[:, 5:10]) > 0)  # spectral leakage from the neighbours


# ---------------------------------------------------------------- GPU

gpu = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def _close(got, want, tol=2e-5):
    got = np.asarray(got, np.complex128)
    want = np.asarray(want, np.complex128)
    scale = np.sqrt(np.mean(np.abs(want) ** 2))
    err = np.abs(got - want).max() / scale
    assert err < tol, f"max |gpu - oracle| / rms = {err:.3g}"
    m = np.abs(want) > 0.05 * scale
    if m.any():
        ph = np.abs(np.angle(got[m] * np.conj(want[m])))
        assert ph.max() < 1e-3, f"max phase error {ph.max():.3g} rad"


@gpu
@pytest.mark.parametrize("na,nd,lac,ldn,scale,mask", [
    (300, 40, 2, 3, 0.5, True), (64, 16, 1, 1, 1.0, False), (257, 9, 4, 2, 2.0, True),
    (1000, 6, 5, 1, 1.0, True),
    # lines of 2,049-4,096 samples: the fused shared-memory upsampling
    (2500, 12, 4, 2, 0.5, True), (4096, 5, 1, 1, 1.0, False), (2049, 4, 3, 1, 2.0, True)])
def test_gpu_crossmul_matches_oracle(torch_cuda, na, nd, lac, ldn, scale, mask):
    torch = torch_cuda
    from srg_b200 import api
    rng = np.random.default_rng(na + nd)
    x, y = _img(rng, nd, na), _img(rng, nd, na)
    y = (0.6 * x + 0.8 * y).astype(np.complex64)  # partly coherent pair
    x[:, na // 3: na // 3 + 2 * lac] = 0           # an empty window for the mask
    want_ig, want_am = ox.crossmul(x, y, looksac=lac, looksdn=ldn, scale=scale, mask=mask)
    ig, am = api.crossmul(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), looksac=lac,
                          looksdn=ldn, scale=scale, mask=mask)
    _close(ig.cpu().numpy(), want_ig)
    _close(am.cpu().numpy(), want_am)
    if mask:
        assert np.array_equal(ig.cpu().numpy() == 0, want_ig == 0)


@gpu
def test_gpu_crossmul_row_stride_and_valid_lines(torch_cuda):
    torch = torch_cuda
    from srg_b200 import api
    rng = np.random.default_rng(7)
    big = _img(rng, 20, 140)
    x, y = big[:, :100], big[:, 20:120]            # row stride 140
    want_ig, want_am = ox.crossmul(x, y, looksac=2, looksdn=2, nvalid=15)
    tb = torch.from_numpy(big).cuda()
    ig, am = api.crossmul(tb[:, :100], tb[:, 20:120], looksac=2, looksdn=2, nvalid=15)
    assert ig.shape == (7, 50)
    _close(ig.cpu().numpy(), want_ig)
    _close(am.cpu().numpy(), want_am)


@gpu
@pytest.mark.parametrize("na,ldn", [(200, 4), (2600, 4), (2600, 1)])
def test_gpu_crossmul_stack_equals_pairs(torch_cuda, na, ldn):
    """A stack's pairs equal the pairs formed one by one (na 2,600 with looks
    of one line down: the fused stack kernel; also against the oracle)."""
    torch = torch_cuda
    from srg_b200 import api
    rng = np.random.default_rng(8)
    hosts = [_img(rng, 24, na) for _ in range(5)]
    hosts[2][:, 500:520] = 0                       # an empty window for the mask
    imgs = [torch.from_numpy(h).cuda() for h in hosts]
    igs, ams = api.crossmul_stack(imgs, looksac=2, looksdn=ldn, scale=0.25, mask=True)
    for k in range(4):
        ig, am = api.crossmul(imgs[k], imgs[k + 1], looksac=2, looksdn=ldn, scale=0.25, mask=True)
        assert torch.equal(ig, igs[k]) and torch.equal(am, ams[k])
        if na > 2048:
            want_ig, want_am = ox.crossmul(hosts[k], hosts[k + 1], looksac=2, looksdn=ldn,
                                           scale=0.25, mask=True)
            _close(igs[k].cpu().numpy(), want_ig)
            _close(ams[k].cpu().numpy(), want_am)


@gpu
def test_gpu_crossmul_long_stack_in_launches(torch_cuda):
    """A stack of 66 images with looks of one line down and 2,100-sample
    lines: the fused stack kernel takes it in two launches of up to 64
    images that share one; every pair equals the pair formed alone."""
    torch = torch_cuda
    from srg_b200 import api
    rng = np.random.default_rng(10)
    imgs = [torch.from_numpy(_img(rng, 6, 2100)).cuda() for _ in range(66)]
    igs, ams = api.crossmul_stack(imgs, looksac=3, looksdn=1, scale=0.5)
    assert len(igs) == 65
    for k in (0, 61, 62, 63, 64):
        ig, am = api.crossmul(imgs[k], imgs[k + 1], looksac=3, looksdn=1, scale=0.5)
        assert torch.equal(ig, igs[k]) and torch.equal(am, ams[k]), k


@gpu
def test_gpu_crossmul_files_matches_oracle(torch_cuda):
    from srg_b200 import crossmul as cm
    rng = np.random.default_rng(9)
    x, y = _img(rng, 30, 90), _img(rng, 30, 90)
    with tempfile.TemporaryDirectory() as td:
        f1, f2, fi, fa = (os.path.join(td, n) for n in ("a.geo", "b.geo", "i.int", "i.amp"))
        x.tofile(f1)
        y.tofile(f2)
        assert cm.main([f1, f2, fi, fa, "90", "28", "1.5", "3", "2"]) == 0
        ig = np.fromfile(fi, np.complex64).reshape(14, 30)
        am = np.fromfile(fa, np.complex64).reshape(14, 30)
    want_ig, want_am = ox.crossmul(x, y, looksac=3, looksdn=2, scale=1.5, nvalid=28)
    _close(ig, want_ig)
    _close(am, want_am)


@gpu
def test_gpu_crossmul_rejects_bad_looks(torch_cuda):
    torch = torch_cuda
    from srg_b200 import _lib, api
    x = torch.zeros((4, 8), dtype=torch.complex64, device="cuda")
    with pytest.raises(_lib.SrgError):
        api.crossmul(x, x, looksac=16, looksdn=1)
