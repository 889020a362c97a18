"""Finer range lines for the backprojection's linear interpolation
(srg_oversample_range_device): the half-sample filter, its output against a
numpy evaluation, its interpolation error on band-limited lines, and the
backprojection of 2x-oversampled point-target data in both forms."""
import numpy as np
import pytest

from srg_b200 import _lib, api, scene


def _np_oversample(x, h):
    P, S = x.shape
    out = np.zeros((P, 2 * S - 1), np.complex128)
    out[:, 0::2] = x
    xp = np.concatenate([np.zeros((P, 3)), x, np.zeros((P, 4))], axis=1)
    for k in range(S - 1):
        acc = 0
        for t in range(4):
            acc = acc + h[t] * (xp[:, 3 + k - t] + xp[:, 3 + k + 1 + t])
        out[:, 2 * k + 1] = acc
    return out


def test_half_sample_taps():
    h = api.oversample_taps().astype(np.float64)
    assert abs(2 * h.sum() - 1.0) < 1e-6            # unit DC gain
    assert np.all(np.sign(h) == [1, -1, 1, -1])     # windowed sinc at 0.5, 1.5, 2.5, 3.5
    assert np.all(np.abs(h[1:]) < np.abs(h[:-1]))


gpu = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


@gpu
def test_gpu_oversample_matches_numpy(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((5, 301)) + 1j * rng.standard_normal((5, 301))).astype(np.complex64)
    h = api.oversample_taps().astype(np.float64)
    want = _np_oversample(x.astype(np.complex128), h)
    tin = torch.from_numpy(x).cuda()
    out = torch.zeros((5, 602), dtype=torch.complex64, device="cuda")
    _lib.check(_lib.lib().srg_oversample_range_device(
        _lib.C.c_void_p(tin.data_ptr()), 301, 5, 301, _lib.C.c_void_p(out.data_ptr()), 602, None))
    torch.cuda.synchronize()
    got = out[:, :601].cpu().numpy()
    assert np.abs(got - want).max() < 1e-5 * np.abs(want).max()
    assert torch.count_nonzero(out[:, 601]).item() == 0


@gpu
def test_gpu_oversample_interpolates_band_limited_lines(torch_cuda):
    # tones up to 0.3 cycles/sample: the half-sample values within 1 % of the
    # truth (linear midpoints miss by ~20 %)
    torch = torch_cuda
    n = np.arange(400)
    f = np.array([0.05, 0.17, 0.3])
    line = sum(np.exp(2j * np.pi * fk * n) for fk in f)[None].astype(np.complex64)
    mid = sum(np.exp(2j * np.pi * fk * (n[:-1] + 0.5)) for fk in f)
    tin = torch.from_numpy(line).cuda()
    out = torch.zeros((1, 800), dtype=torch.complex64, device="cuda")
    _lib.check(_lib.lib().srg_oversample_range_device(
        _lib.C.c_void_p(tin.data_ptr()), 400, 1, 400, _lib.C.c_void_p(out.data_ptr()), 800, None))
    torch.cuda.synchronize()
    odd = out[0, 1:799:2].cpu().numpy()
    inner = slice(8, 391)  # away from the zero-padded ends
    err = np.abs(odd[inner] - mid[inner]).max() / 3.0
    lin = np.abs(0.5 * (line[0, :-1] + line[0, 1:])[inner] - mid[inner]).max() / 3.0
    assert err < 0.01 and lin > 0.1, (err, lin)


@gpu
def test_gpu_backprojection_of_oversampled_lines(torch_cuda):
    torch = torch_cuda
    b = scene.config0_point_targets(seed=1000, pulses=1024, samples=4096, ntargets=24)
    db = api.to_device(b)
    peaks = {}
    outs = {}
    for name, burst in (("plain", db), ("x2", api.oversample2(db))):
        for form in (_lib.FORM_FP64, _lib.FORM_SPLIT):
            api.backproject([burst], form=form)
            outs[(name, form)] = db.out.clone().cpu().numpy()
    tl = b.targets[:, 0].astype(int) - db.firstline
    tp = b.targets[:, 1].astype(int)
    for name in ("plain", "x2"):
        peaks[name] = np.abs(outs[(name, _lib.FORM_FP64)][tl, tp])
        # split vs FP64 on the same lines: far inside the 1 mrad budget
        s, d = outs[(name, _lib.FORM_SPLIT)], outs[(name, _lib.FORM_FP64)]
        a = np.abs(d)
        m = a > 0.05 * np.sqrt(np.mean(a[a > 0] ** 2))
        ph = np.angle(s[m] * np.conj(d[m])) * 1e3
        assert np.sqrt(np.mean(ph ** 2)) < 1.0
    # the finer line loses less to linear interpolation at the focused peaks
    assert np.mean(peaks["x2"]) > np.mean(peaks["plain"])
    # and the focused phase of each target agrees between the two lines
    dphi = np.angle(outs[("x2", _lib.FORM_FP64)][tl, tp] * np.conj(outs[("plain", _lib.FORM_FP64)][tl, tp]))
    assert np.abs(dphi).max() < 0.05
