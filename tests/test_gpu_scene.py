"""Scene plans (srg_scene_*): batched azimuth centres, one persistent
backprojection launch for several bursts, ordered merge into a scene raster
and CUDA-graph replay, against the oracle merging the bursts one by one."""
import numpy as np
import pytest

import oracle as O
from helpers import phase_amp_errors, rel_err
from srg_b200 import _lib, api, scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


@pytest.fixture(scope="module")
def mini():
    grid, bursts = scene.mini_scene()
    orc = O.Oracle()
    geo = np.zeros((grid.length, grid.width), np.complex64)
    terms = 0
    for b in bursts:
        geo, t = orc.burst_geo(b, geo=geo, gpu=True)
        terms += t
    return grid, bursts, geo, terms


def build(torch, grid, bursts, form, tile_cfg=-1, tile_shear=None):
    dem = torch.from_numpy(grid.dem).cuda()
    dbs = [api.to_device(b, dem_tensor=dem, narrow_out=True) for b in bursts]
    raster = torch.zeros((grid.length, grid.width), dtype=torch.complex64, device="cuda")
    return dbs, raster, api.Scene(dbs, raster=raster, form=form, tile_cfg=tile_cfg,
                                  tile_shear=tile_shear)


WS_FP64 = [c[0] for c in _lib.tile_configs()
           if c[1] == _lib.FORM_FP64 and _lib.tile_config_name(c[0]).startswith("bp_ws")]


@pytest.mark.parametrize("shear", [None, -3])
@pytest.mark.parametrize("form", [_lib.FORM_FP64, _lib.FORM_SPLIT])
def test_scene_plan_matches_sequential_merge(torch_cuda, mini, form, shear):
    """The plan's passes (graph replays and direct launches) against the
    oracle's bursts merged one after the other; with sheared tiles the merge
    reads the work-list mask along the shear."""
    torch = torch_cuda
    grid, bursts, geo, terms = mini
    assert geo.any()
    cfg = WS_FP64[0] if (shear is not None and form == _lib.FORM_FP64) else -1
    dbs, raster, sc = build(torch, grid, bursts, form, cfg, shear)
    assert sc.terms() == terms
    st = torch.cuda.Stream()
    for rep in range(3):          # first pass captures the graph, then replays
        raster.zero_()
        for db in dbs:            # every burst pixel is written by the pass, formed or not
            db.out.fill_(complex(7.0, 7.0))
        sc.run(st.cuda_stream)
        sc.sync(st.cuda_stream)
        for db in dbs:
            assert not bool((db.out == complex(7.0, 7.0)).any())
        got = raster.cpu().numpy()
        assert np.array_equal(got != 0, geo != 0)
        if form == _lib.FORM_FP64:
            assert rel_err(got, geo) < 2e-6
        else:
            e = phase_amp_errors(got, geo)
            assert e["ph_rms"] < 1.0 and e["amp_rms"] < 1e-3, e
    # default stream: direct launches, same result
    raster.zero_()
    sc.run(0)
    sc.sync(0)
    assert np.array_equal(raster.cpu().numpy().view(np.uint32), got.view(np.uint32))
    sc.close()


def test_scene_tune_picks_a_valid_shape(torch_cuda, mini):
    torch = torch_cuda
    grid, bursts, geo, _ = mini
    dbs, raster, sc = build(torch, grid, bursts, _lib.FORM_SPLIT)
    cfg, ms = sc.tune(iters=2)
    assert _lib.tile_configs()[cfg][1] == _lib.FORM_SPLIT and ms > 0
    assert sc.shape() == cfg
    sc.run(0)
    sc.sync(0)
    e = phase_amp_errors(raster.cpu().numpy(), geo)
    assert e["ph_rms"] < 1.0, e
    sc.close()


def test_scene_rejects_precomputed_coefficients(torch_cuda, mini):
    torch = torch_cuda
    grid, bursts, _, _ = mini
    db = api.to_device(bursts[0])
    coef = api.line_centres(db)
    d = (api.BurstDesc * 1)(db.desc(coef.data_ptr()))
    import ctypes as C
    h = C.c_void_p()
    rc = _lib.lib().srg_scene_create(d, 1, None, 0, 0, 0, None, C.byref(h))
    assert rc == _lib.SRG_E_ARG and "coef must be NULL" in _lib.last_error()
