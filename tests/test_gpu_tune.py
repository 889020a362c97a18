"""The autotuner's search: the range interpolation (the original lines, or
2x-oversampled ones) chosen against a phase-error budget from the lines'
own spectrum, the kernel shape timed or taken from the results cache, and
the cache carried to a later process through SRG_TUNE_CACHE."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from srg_b200 import _lib, api, scene

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def band_limited(rng, nlines, n, band):
    """Periodic complex lines of n samples, white within |nu| < band."""
    nu = np.fft.fftfreq(n)
    spec = (rng.standard_normal((nlines, n)) + 1j * rng.standard_normal((nlines, n)))
    spec[:, np.abs(nu) >= band] = 0
    return spec, nu


def measured(spec, nu, taps):
    """Direct RMS phase error (relative error / sqrt 2) of linear interpolation
    on the lines and on their 2x-oversampled version, over offsets u."""
    x = np.fft.ifft(spec, axis=1)
    power = np.mean(np.abs(x) ** 2)
    el, eo, cnt = 0.0, 0.0, 0
    y = sum(taps[t] * (np.roll(x, t, axis=1) + np.roll(x, -1 - t, axis=1)) for t in range(4))
    for u in (np.arange(16) + 0.5) / 16:
        at = lambda s: np.fft.ifft(spec * np.exp(2j * np.pi * nu * s), axis=1)  # noqa: E731
        xn1 = np.roll(x, -1, axis=1)
        el += np.mean(np.abs((1 - u) * x + u * xn1 - at(u)) ** 2)
        eo += 0.5 * np.mean(np.abs((1 - u) * x + u * y - at(u / 2)) ** 2)
        eo += 0.5 * np.mean(np.abs((1 - u) * y + u * xn1 - at((1 + u) / 2)) ** 2)
        cnt += 1
    return np.sqrt(el / cnt / power / 2), np.sqrt(eo / cnt / power / 2)


@pytest.mark.parametrize("band", [0.44, 0.25])
def test_interp_error_estimate_matches_direct_measurement(torch_cuda, band):
    torch = torch_cuda
    rng = np.random.default_rng(5)
    spec, nu = band_limited(rng, 32, 4096, band)
    lines = np.fft.ifft(spec, axis=1).astype(np.complex64)
    el, eo = api.interp_error(torch.from_numpy(lines).cuda(), sample_lines=32)
    ml, mo = measured(spec, nu, api.oversample_taps().astype(np.float64))
    assert abs(el - ml) < 0.05 * ml, (el, ml)
    assert abs(eo - mo) < 0.05 * mo + 1e-4, (eo, mo)
    assert eo < 0.75 * el


def _mini_plan(torch, form=_lib.FORM_SPLIT):
    grid, bursts = scene.mini_scene()
    dem = torch.from_numpy(grid.dem).cuda()
    dbs = [api.to_device(b, dem_tensor=dem, narrow_out=True) for b in bursts]
    return dbs, api.Scene(dbs, raster=None, form=form)


def test_autotune_interpolation_budget_and_cache(torch_cuda):
    torch = torch_cuda
    dbs, sc = _mini_plan(torch)
    r = sc.autotune(interp_budget=10.0, iters=1, use_cache=False)   # anything goes: linear
    assert r["interp"] == _lib.INTERP_LINEAR and r["from_cache"] == 0 and r["ms"] > 0
    assert r["tile_shear"] in (0, _lib.TILE_SHEAR_AUTO)
    assert r["err_linear"] > r["err_oversampled"] > 0
    # a second plan of the same shape takes the cached shape without timing
    # shapes; it times the shear only where the geometric one shears a burst
    dbs2, sc2 = _mini_plan(torch)
    r2 = sc2.autotune(iters=1)
    assert r2["from_cache"] == 1 and r2["tile_cfg"] == r["tile_cfg"]
    geo = False
    for db in dbs2:
        sh, tx, ty = C.c_int(), C.c_int(), C.c_int()
        d = db.desc()
        assert _lib.lib().srg_tile_shear(C.byref(d), r["tile_cfg"], _lib.TILE_SHEAR_AUTO,
                                         C.byref(sh), C.byref(tx), C.byref(ty)) == _lib.SRG_OK
        geo |= sh.value != 0
    assert (r2["ms"] == -1) == (not geo)
    # a budget below the linear error: oversampled lines, made by the plan in
    # every pass; the images equal a plan's on lines oversampled beforehand
    r3 = sc.autotune(interp_budget=0.5 * r["err_linear"], iters=1, use_cache=False)
    assert r3["interp"] == _lib.INTERP_OVERSAMPLED2 and sc.interp() == _lib.INTERP_OVERSAMPLED2
    st = torch.cuda.Stream()
    sc.run(st.cuda_stream)
    sc.sync(st.cuda_stream)
    got = [db.out.clone() for db in dbs]
    over = [api.oversample2(db) for db in dbs2]
    ref_plan = api.Scene(over, raster=None, form=_lib.FORM_SPLIT, tile_cfg=r3["tile_cfg"],
                         tile_shear=r3["tile_shear"])
    ref_plan.run(st.cuda_stream)
    ref_plan.sync(st.cuda_stream)
    for g, db in zip(got, over):
        assert torch.equal(g.view(torch.float32), db.out.view(torch.float32))
    assert sc.terms() == ref_plan.terms()
    # back to the original lines
    sc.set_interp(_lib.INTERP_LINEAR)
    assert sc.interp() == _lib.INTERP_LINEAR
    for p in (sc, sc2, ref_plan):
        p.close()


CHILD = r"""
import json, sys, torch
sys.path.insert(0, sys.argv[1])
from srg_b200 import _lib, api, scene
grid, bursts = scene.mini_scene(seed=int(sys.argv[2]))
dem = torch.from_numpy(grid.dem).cuda()
dbs = [api.to_device(b, dem_tensor=dem, narrow_out=True) for b in bursts]
sc = api.Scene(dbs, raster=None, form=_lib.FORM_FP64)
print(json.dumps(sc.autotune(iters=1)))
"""


def test_tune_cache_file_carries_to_another_process(torch_cuda, tmp_path):
    env = dict(os.environ, SRG_TUNE_CACHE=str(tmp_path / "tune.txt"))
    outs = []
    for _ in range(2):
        p = subprocess.run([sys.executable, "-c", CHILD, ROOT, "77"], env=env, capture_output=True,
                           text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        outs.append(json.loads(p.stdout.strip().splitlines()[-1]))
    assert outs[0]["from_cache"] == 0 and outs[1]["from_cache"] == 1
    assert outs[0]["tile_cfg"] == outs[1]["tile_cfg"]
    assert (tmp_path / "tune.txt").read_text().count("\n") == 1
