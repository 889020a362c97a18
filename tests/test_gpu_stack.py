"""Repeat-pass chain on the GPU: two passes with a perpendicular baseline
and an along-track shift, a known line-of-sight motion of isolated point
targets between them, forward projection -> backprojection (both forms) ->
crossmul.  The interferogram phase at every target must be the injected
4 pi / lambda * (range change), whatever the baseline (the backprojection
removes the whole geometric phase of each pass)."""
import numpy as np
import pytest

from srg_b200 import _lib, api, scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def _targets(b, n, rng):
    ok = scene.formed_mask_estimate(b, margin=24)
    ok[:, :10] = ok[:, -10:] = False
    ok[:10] = ok[-10:] = False
    cand = np.argwhere(ok)
    chosen = []
    for i in rng.permutation(len(cand)):
        y, x = cand[i]
        if all(max(abs(y - cy), abs(x - cx)) >= 12 for cy, cx in chosen):
            chosen.append((y, x))
            if len(chosen) == n:
                break
    return np.array(chosen)


def test_stack_interferogram_recovers_injected_motion(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(44)
    base = scene.make_geometry(pulses=1024, samples=4096, width=256, length=256, spacing=0.0002,
                               centre_height=500.0)
    base.dem = np.full((256, 256), 500, np.int16)
    e_perp, speed = scene.baseline_frame(base)
    # smooth motion field: up to 2 cm of range change (0.45 rad of phase)
    drange = scene.mogi_range_change(base, depth=3000.0, los_max=0.02)
    pick = _targets(base, 16, rng)
    assert len(pick) >= 8
    refl = torch.zeros((256, 256), dtype=torch.complex64, device="cuda")
    refl[torch.from_numpy(pick[:, 0]).cuda(), torch.from_numpy(pick[:, 1]).cuda()] = 1.0
    dem_t = torch.from_numpy(base.dem).cuda()
    outs = {f: [] for f in (_lib.FORM_FP64, _lib.FORM_SPLIT)}
    for k, (bp, al) in enumerate([(0.0, 0.0), (110.0, 2.5)]):
        b = scene.make_geometry(pulses=1024, samples=4096, width=256, length=256, spacing=0.0002,
                                centre_height=500.0, grid_centre=scene.grid_centre(base),
                                position_offset=bp * e_perp, along_offset=al / speed)
        b.firstlat, b.firstlon, b.latlons = base.firstlat, base.firstlon, base.latlons.copy()
        b.dem = base.dem
        bt = torch.zeros((1024, 4096), dtype=torch.complex64, device="cuda")
        db = api.to_device(b, burst_tensor=bt, dem_tensor=dem_t)
        assert db.firstline == 0 and db.nlines == 256
        offs = torch.from_numpy(drange * float(k)).cuda().contiguous()
        satvel = torch.from_numpy(np.ascontiguousarray(b.satvel)).cuda()
        api.forward_project(db, refl, satvel, range_offset=offs)
        torch.cuda.synchronize()
        for f in outs:
            api.backproject([db], form=f)
            outs[f].append(db.out.clone())
    want = 4.0 * np.pi / base.wvl * drange[pick[:, 0], pick[:, 1]]
    assert np.abs(want).max() > 0.1  # the motion is visible
    for f, (a, b) in outs.items():
        ig, _ = api.crossmul(a, b, looksac=1, looksdn=1, mask=False)
        got = ig.cpu().numpy()[pick[:, 0], pick[:, 1]]
        err = np.angle(got * np.exp(-1j * want))
        assert np.abs(err).max() < 5e-3, (f, err)
    # split vs FP64 interferograms agree far inside the 1 mrad budget
    igs, _ = api.crossmul(*outs[_lib.FORM_SPLIT], mask=False)
    igd, _ = api.crossmul(*outs[_lib.FORM_FP64], mask=False)
    s = igs.cpu().numpy()[pick[:, 0], pick[:, 1]]
    d = igd.cpu().numpy()[pick[:, 0], pick[:, 1]]
    assert np.abs(np.angle(s * np.conj(d))).max() < 1e-3
