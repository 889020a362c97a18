"""Parity of the CUDA path (libsrg_bp.so, called through its C ABI) with the
oracle and the golden fixtures made by the compiled reference."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from helpers import MINI_CASES, load_golden, mini_case, phase_amp_errors, rel_err
from srg_b200 import _lib, api, scene

pytestmark = pytest.mark.gpu
NAMES = [c[0] for c in MINI_CASES]
SPLIT_CFGS = [c[0] for c in _lib.tile_configs() if c[1] == _lib.FORM_SPLIT]
FP64_CFGS = [c[0] for c in _lib.tile_configs() if c[1] == _lib.FORM_FP64]
# the warp-specialised FP64 shapes (they take sheared tiles)
WS_FP64_CFGS = [c for c in FP64_CFGS if _lib.tile_config_name(c).startswith("bp_ws")]
SHAPES = {c[0]: c for c in _lib.tile_configs()}


def shear_fits(cfg, shear):
    """A shear offsets a tile's columns by fewer lines than it is tall."""
    tx, ty = SHAPES[cfg][2], SHAPES[cfg][3]
    return abs((shear * (tx - 1)) // 32) < ty

# Tolerances.  FP64 form vs the oracle's GPU form: identical bins, weights and
# phases up to the last ulp of sin/cos and of the FP64 accumulation order, so
# the complex64 outputs agree to FP32 rounding.  Split form: the acceptance
# bound of the design (<= 1 mrad RMS phase error against the FP64 oracle),
# with the measured errors ~100x smaller.
FP64_REL = 2e-6
SPLIT_PH_RMS_MRAD = 1.0
SPLIT_PH_MAX_MRAD = 10.0
SPLIT_AMP_RMS = 1e-3


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


@pytest.fixture(scope="module")
def orc():
    O.build()
    return O.Oracle()


def run_dev(b, form, cfg=-1):
    db = api.to_device(b)
    api.backproject([db], form=form, tile_cfg=cfg)
    return db, db.out.cpu().numpy()


def oracle_gpu_form(orc, b):
    return orc.stages(b, gpu_lerp=1, gpu_scale=1, want_acc=True)


@pytest.mark.parametrize("name", NAMES)
def test_line_centres_exact(torch_cuda, orc, name):
    b = mini_case(name)
    st = orc.stages(b)
    db = api.to_device(b)
    coef = api.line_centres(db).cpu().numpy()
    assert np.array_equal(coef, st["coef"])


@pytest.mark.parametrize("name", NAMES)
def test_term_count_exact(torch_cuda, orc, name):
    b = mini_case(name)
    st = orc.stages(b)
    db = api.to_device(b)
    assert api.count_terms([db]) == st["terms"]


@pytest.mark.parametrize("cfg", FP64_CFGS)
@pytest.mark.parametrize("name", NAMES)
def test_fp64_form_matches_oracle(torch_cuda, orc, name, cfg):
    b = mini_case(name)
    st = oracle_gpu_form(orc, b)
    _, out = run_dev(b, _lib.FORM_FP64, cfg)
    ref = st["out"]
    assert np.array_equal(out != 0, ref != 0)
    assert rel_err(out, ref) < FP64_REL


@pytest.mark.parametrize("cfg", SPLIT_CFGS)
@pytest.mark.parametrize("name", NAMES)
def test_split_form_within_phase_budget(torch_cuda, orc, name, cfg):
    b = mini_case(name)
    st = oracle_gpu_form(orc, b)
    _, out = run_dev(b, _lib.FORM_SPLIT, cfg)
    e = phase_amp_errors(out, st["out"])
    assert e["n"] > 100
    assert e["ph_rms"] < SPLIT_PH_RMS_MRAD, e
    assert e["ph_max"] < SPLIT_PH_MAX_MRAD, e
    assert e["amp_rms"] < SPLIT_AMP_RMS, e


@pytest.mark.parametrize("name", NAMES)
def test_fp64_form_matches_golden_reference(torch_cuda, name):
    """Against the compiled reference's own raw sums (CPU form: unscaled, FP64
    interpolation), rescaled by the aperture length."""
    b, g = load_golden(name)
    _, out = run_dev(b, _lib.FORM_FP64)
    az = g["ref_azoff"]
    a0 = np.clip(np.round(az - b.aperture // 2).astype(int), 0, None)
    a1 = np.clip(np.round(az + b.aperture // 2).astype(int), None, b.rawdatalines - 1)
    formed = az > 0
    ref = np.zeros_like(g["ref_pixelint"])
    ref[formed] = g["ref_pixelint"][formed] * (1.0 / (a1 - a0)[formed]).astype(np.float32)
    assert rel_err(out, ref) < 1e-5


@pytest.mark.parametrize("form", [_lib.FORM_FP64, _lib.FORM_SPLIT])
@pytest.mark.parametrize("name", ["slope", "inset", "oddS"])
def test_dropin_entry_matches_oracle_entry(torch_cuda, orc, name, form):
    """azimuth_compress_ (33 by-reference arguments, DEM and .geo by file
    descriptor) against the oracle's entry with the GPU merge rule, starting
    from a non-zero .geo so that the merge rule is exercised."""
    b = mini_case(name)
    rng = np.random.default_rng(7)
    init = (rng.standard_normal((b.demlength, b.demwidth)) +
            1j * rng.standard_normal((b.demlength, b.demwidth))).astype(np.complex64)
    ref = O.run_33_files(orc.lib.srg_oracle_azimuth_compress_, b, geo_init=init)
    api.set_default_form(form)
    try:
        got = O.run_33_files(_lib.lib().azimuth_compress_, b, geo_init=init)
    finally:
        api.set_default_form(_lib.FORM_SPLIT)
    changed_ref = ref != init
    changed = got != init
    assert np.array_equal(changed, changed_ref)
    if form == _lib.FORM_FP64:
        assert rel_err(got, ref) < FP64_REL
    else:
        e = phase_amp_errors(got[changed], ref[changed])
        assert e["ph_rms"] < SPLIT_PH_RMS_MRAD, e


def test_dropin_pinned_upload_in_blocks(torch_cuda):
    """With the range lines in pinned host memory the drop-in starts the
    backprojection while the lines are still uploading (block by block, each
    chunk waiting for its rows); the .geo it writes is bit-identical to the
    one from pageable lines (uploaded in full before the launch), call after
    call."""
    torch = torch_cuda
    b = scene.config0_point_targets()
    pinned = torch.from_numpy(np.ascontiguousarray(b.burst, np.complex64)).pin_memory()
    outs = []
    with tempfile.TemporaryDirectory() as td:
        dem_path = os.path.join(td, "e.dem")
        np.ascontiguousarray(b.dem, np.int16).tofile(dem_path)
        fd_dem = os.open(dem_path, os.O_RDWR)
        try:
            for i, host in enumerate([b.burst, pinned.numpy(), pinned.numpy(), b.burst]):
                geo_path = os.path.join(td, f"s{i}.geo")
                np.zeros((b.demlength, b.demwidth), np.complex64).tofile(geo_path)
                fd = os.open(geo_path, os.O_RDWR)
                try:
                    api.azimuth_compress_files(b, fd, fd_dem, burst=host)
                finally:
                    os.close(fd)
                outs.append(np.fromfile(geo_path, np.complex64))
        finally:
            os.close(fd_dem)
    assert np.count_nonzero(outs[0]) > 0
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))


def test_status_entry_reports_errors(torch_cuda):
    b = mini_case("flat")
    with tempfile.TemporaryDirectory() as td:
        dem = os.path.join(td, "d.dem")
        b.dem.astype(np.int16).tofile(dem)
        fd = os.open(dem, os.O_RDONLY)
        try:
            with pytest.raises(_lib.SrgError) as ei:
                # output descriptor -1: the DEM is read, the .geo read fails
                api.azimuth_compress_status(b, -1, fd, form=_lib.FORM_SPLIT)
            assert ei.value.code == _lib.SRG_E_IO
        finally:
            os.close(fd)


def test_batched_launch_equals_single(torch_cuda):
    bs = [mini_case(n) for n in ("flat", "tops", "inset", "oddS")]
    singles = [run_dev(b, _lib.FORM_SPLIT)[1] for b in bs]
    dbs = [api.to_device(b) for b in bs]
    api.backproject(dbs, form=_lib.FORM_SPLIT)
    for db, s in zip(dbs, singles):
        assert np.array_equal(db.out.cpu().numpy().view(np.uint32), s.view(np.uint32))


def test_pulse_orbit_kernel(torch_cuda, orc):
    """Per-pulse orbit on the GPU against the oracle's restatement of
    sentinel/sentineltimingsub.f90:41,55-63 (window from the truncated index,
    unclamped, orbithermite.f): bit for bit; and against the orbit the
    state vectors were sampled from."""
    torch = torch_cuda
    b = scene.make_geometry(pulses=1500, samples=64, width=8, length=8, spacing=1e-4,
                            quantise=False)
    t = torch.from_numpy(b.pulse_time).cuda()
    pos, vel = api.pulse_orbit(t, b)
    opos, ovel = orc.pulse_orbit(b.pulse_time, b)
    assert np.array_equal(pos.cpu().numpy(), opos)
    assert np.array_equal(vel.cpu().numpy(), ovel)
    np.testing.assert_allclose(pos.cpu().numpy(), b.satloc, rtol=0, atol=1e-6)
    np.testing.assert_allclose(vel.cpu().numpy(), b.satvel, rtol=0, atol=1e-9)


def test_config0_point_targets(torch_cuda, orc):
    """Configuration 0: 1,024 x 4,096 burst, 64 point targets, 256 x 256 grid.
    Both forms against the oracle, and the physics check: every target focuses
    on its own pixel with a phase near zero."""
    b = scene.config0_point_targets()
    st = oracle_gpu_form(orc, b)
    db = api.to_device(b)
    assert api.count_terms([db]) == st["terms"]
    api.backproject([db], form=_lib.FORM_FP64)
    f64 = db.out.cpu().numpy()
    assert rel_err(f64, st["out"]) < FP64_REL
    api.backproject([db], form=_lib.FORM_SPLIT)
    spl = db.out.cpu().numpy()
    e = phase_amp_errors(spl, st["out"])
    assert e["ph_rms"] < SPLIT_PH_RMS_MRAD and e["amp_rms"] < SPLIT_AMP_RMS, e
    fl = st["firstline"]
    for line, pix, _ in b.targets.astype(int):
        li = line - fl
        assert st["azoff"][li, pix] > 0
        win = np.abs(spl[li - 2:li + 3, pix - 2:pix + 3])
        assert np.unravel_index(np.argmax(win), win.shape) == (2, 2)
        assert abs(np.angle(spl[li, pix])) < 0.1


@pytest.mark.parametrize("shear", [None, -3, 4])
@pytest.mark.parametrize("form", [_lib.FORM_FP64, _lib.FORM_SPLIT])
def test_tiles_without_formed_pixels(torch_cuda, orc, form, shear):
    """A grid reaching far past the lines the pulses see: most tiles hold no
    formed pixel and stay out of the kernel's work list.  Their pixels still
    come out zero (the output starts filled with 7+7j) and the formed pixels
    match the oracle; with sheared tiles too (forced on the warp-specialised
    shapes, whose dropped tiles are zeroed line by line along the shear)."""
    b = scene.mini_fixture(seed=31, length=400, width=96)
    ref = oracle_gpu_form(orc, b)["out"]
    rows = np.abs(ref).sum(axis=1) > 0
    assert 0 < rows.sum() < 0.5 * len(rows)          # mostly unformed lines
    db = api.to_device(b)
    db.out.fill_(complex(7.0, 7.0))
    cfg = WS_FP64_CFGS[0] if (shear is not None and form == _lib.FORM_FP64) else -1
    api.backproject([db], form=form, tile_cfg=cfg, tile_shear=shear)
    out = db.out.cpu().numpy()
    assert not np.any(out == np.complex64(7 + 7j))
    assert np.array_equal(out != 0, ref != 0)
    if form == _lib.FORM_FP64:
        assert rel_err(out, ref) < FP64_REL
    else:
        e = phase_amp_errors(out, ref)
        assert e["ph_rms"] < SPLIT_PH_RMS_MRAD and e["amp_rms"] < SPLIT_AMP_RMS, e


@pytest.mark.parametrize("shear", [-7, -3, 4])
@pytest.mark.parametrize("name", NAMES)
def test_sheared_tiles_match_oracle(torch_cuda, orc, name, shear):
    """Tiles sheared by `shear` columns per grid line (forced: the mini grids
    are too narrow for the geometric choice to take a shear).  The FP64 form
    on the warp-specialised shapes gives every pixel the same terms in the
    same pulse order as rectangular tiles, so the outputs agree with those and
    with the oracle to FP32 rounding; the split form stays within its budget.
    Every pixel of the burst's columns is written (the output starts filled
    with 7+7j), and no other."""
    b = mini_case(name)
    ref = oracle_gpu_form(orc, b)["out"]
    db = api.to_device(b)
    cols = slice(db.firstpix - db.out_pix0, min(db.lastpix, b.demwidth - 1) - db.out_pix0 + 1)
    for cfg in [c for c in WS_FP64_CFGS if shear_fits(c, shear)]:
        outs = []
        for s in (0, shear):
            db.out.fill_(complex(7.0, 7.0))
            api.backproject([db], form=_lib.FORM_FP64, tile_cfg=cfg, tile_shear=s)
            outs.append(db.out.cpu().numpy())
        rect, sheared = outs
        unset = sheared == np.complex64(7 + 7j)
        assert np.array_equal(unset, rect == np.complex64(7 + 7j))
        assert not np.any(unset[:, cols])
        rect, sheared = np.where(unset, 0, rect), np.where(unset, 0, sheared)
        assert np.array_equal(sheared != 0, ref != 0)
        assert rel_err(sheared, ref) < FP64_REL
        assert rel_err(sheared, rect) < FP64_REL
    db.out.fill_(complex(7.0, 7.0))
    api.backproject([db], form=_lib.FORM_SPLIT, tile_shear=shear)
    out = db.out.cpu().numpy()
    assert np.array_equal(out == np.complex64(7 + 7j), unset)
    out = np.where(unset, 0, out)
    assert np.array_equal(out != 0, ref != 0)
    e = phase_amp_errors(out, ref)
    assert e["ph_rms"] < SPLIT_PH_RMS_MRAD and e["ph_max"] < SPLIT_PH_MAX_MRAD, e
    assert e["amp_rms"] < SPLIT_AMP_RMS, e


def test_dropin_sequential_bursts_merge_like_the_oracle(torch_cuda, orc):
    """Three bursts over one grid and one DEM (different samples and
    apertures, so their formed line bands overlap without coinciding), merged
    in call order into one .geo file through azimuth_compress_ (the scene
    loop of backprojectgpusub.f90): the same file as the oracle's entry
    called the same way (later bursts overwrite earlier ones)."""
    base = mini_case("slope")
    bursts = [base]
    for seed, ap in ((21, 64), (22, 160)):
        b = scene.mini_fixture(seed=seed, dem_kind="slope", aperture=ap)
        b.dem = base.dem
        bursts.append(b)
    rng = np.random.default_rng(5)
    init = (rng.standard_normal((base.demlength, base.demwidth)) +
            1j * rng.standard_normal((base.demlength, base.demwidth))).astype(np.complex64)

    def run(fn):
        with tempfile.TemporaryDirectory() as td:
            dem_path, geo_path = os.path.join(td, "e.dem"), os.path.join(td, "s.geo")
            np.ascontiguousarray(base.dem, np.int16).tofile(dem_path)
            init.tofile(geo_path)
            fd_dem, fd_geo = os.open(dem_path, os.O_RDWR), os.open(geo_path, os.O_RDWR)
            try:
                for b in bursts:
                    O.call_33(fn, b, fd_geo, fd_dem)
                    import ctypes
                    ctypes.CDLL(None).fflush(None)
            finally:
                os.close(fd_dem)
                os.close(fd_geo)
            return np.fromfile(geo_path, np.complex64).reshape(base.demlength, base.demwidth)

    ref = run(orc.lib.srg_oracle_azimuth_compress_)
    api.set_default_form(_lib.FORM_FP64)
    try:
        got = run(_lib.lib().azimuth_compress_)
    finally:
        api.set_default_form(_lib.FORM_SPLIT)
    assert np.array_equal(got != init, ref != init)
    assert (ref != init).sum() > 0
    assert rel_err(got, ref) < FP64_REL


@pytest.mark.parametrize("form", [_lib.FORM_FP64, _lib.FORM_SPLIT])
def test_dropin_with_burst_params_from_line_headers(torch_cuda, orc, form):
    """The caller's side of the call, as backprojectgpusub.f90:140-247 makes
    it: the burst's scalars (PRF, near range, sampling rate, wavelength,
    steering fit angc0/angc1, aperture, limits) derived from the line headers
    and velocities by srg_burst_params, the 10 header samples then zeroed
    (:191), and the call made through azimuth_compress_; the same arguments
    through the oracle's entry give the same .geo."""
    b = mini_case("slope")
    P = b.burst.shape[0]
    pri_code, swst_code = scene.header_codes(b.prf, b.rngstart)
    rng = np.random.default_rng(17)
    addr = np.rint((np.linspace(-0.3, 0.3, P) + 0.9) / 1.8 * 1024).astype(np.int64)
    addr += rng.integers(-2, 3, P)
    lines = b.burst.copy()
    lines[:, :10] = scene.encode_line_headers(b.pulse_time, pri_code, 9, swst_code, 8, addr)
    p = api.burst_params(lines, b.satvel)
    lines[:, :10] = 0
    for k in ("prf", "angc0", "angc1", "rngstart", "rngend", "dmrg", "wvl", "tstart", "tend",
              "tmid", "dtaz", "aperture"):
        setattr(b, k, p[k])
    b.burst = lines
    init = (rng.standard_normal((b.demlength, b.demwidth)) +
            1j * rng.standard_normal((b.demlength, b.demwidth))).astype(np.complex64)
    ref = O.run_33_files(orc.lib.srg_oracle_azimuth_compress_, b, geo_init=init)
    api.set_default_form(form)
    try:
        got = O.run_33_files(_lib.lib().azimuth_compress_, b, geo_init=init)
    finally:
        api.set_default_form(_lib.FORM_SPLIT)
    changed = ref != init
    assert changed.sum() > 1000
    assert np.array_equal(got != init, changed)
    if form == _lib.FORM_FP64:
        assert rel_err(got, ref) < FP64_REL
    else:
        e = phase_amp_errors(got[changed], ref[changed])
        assert e["ph_rms"] < SPLIT_PH_RMS_MRAD, e
