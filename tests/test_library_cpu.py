"""The C ABI library without a GPU: it loads, exports every entry point that
include/srg_bp.h declares, and reports its kernel shapes.  No compute call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from srg_b200 import _lib, api, build, scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "srg_bp.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:srg_\w+|azimuth_compress_\w*))\s*\(", txt)))


def test_library_builds_and_exports_every_declared_symbol():
    build.build()
    L = _lib.lib()
    names = header_functions()
    assert "azimuth_compress_" in names and "srg_bp_bursts_device" in names
    for n in names:
        assert hasattr(L, n), f"{n} declared in srg_bp.h but not exported"


def test_tile_shapes_are_valid():
    cfgs = _lib.tile_configs()
    assert any(c[1] == _lib.FORM_SPLIT for c in cfgs)
    assert any(c[1] == _lib.FORM_FP64 for c in cfgs)
    for idx, form, tx, ty, nt, ck, wb in cfgs:
        assert nt % 32 == 0 and tx % 8 == 0 and ty % 4 == 0
        assert 1 <= ck <= 32
        assert wb % 2 == 0 and 2 <= wb <= 256  # TMA box limits; 16-byte rows
        assert ck * wb * 8 + ck * 48 <= 227 * 1024


def test_default_options():
    o = _lib.default_options()
    assert o.form == _lib.FORM_SPLIT and o.tile_cfg == -1 and o.device == -1


def test_limits_match_oracle():
    import oracle as O
    orc = O.Oracle()
    for name, kw in [("a", dict(seed=1)), ("b", dict(seed=2, latlons_inset=7))]:
        b = scene.mini_fixture(**kw)
        assert api.limits(b) == orc.limits(b)


def test_errors_are_reported_without_gpu_work():
    """Argument validation happens before any device call."""
    import ctypes as C
    L = _lib.lib()
    rc = L.srg_bp_bursts_device(None, 0, None, None)
    assert rc == _lib.SRG_E_ARG
    assert "no bursts" in _lib.last_error()


def _dropin_files(tmp_path, b):
    dem = tmp_path / "d.dem"
    geo = tmp_path / "s.geo"
    np.ascontiguousarray(b.dem, np.int16).tofile(dem)
    init = np.full((b.demlength, b.demwidth), 3 + 4j, np.complex64)
    init.tofile(geo)
    return str(dem), str(geo), init


@pytest.mark.parametrize("field,where", [("xx", "xx"), ("satloc", "satloc"), ("vv", "vv"),
                                         ("rngend", "a scalar argument"), ("latlons", "latlons")])
def test_dropin_refuses_non_finite_geometry_before_any_work(tmp_path, field, where):
    """A NaN or infinity in the orbit, the pulse positions, the box or a
    scalar would leave every pixel unformed without a word (NaN fails every
    window and range test): the status entry refuses it before touching the
    GPU or the files."""
    b = scene.mini_fixture(seed=11)
    v = getattr(b, field)
    if isinstance(v, np.ndarray):
        v = v.copy()
        v.flat[v.size // 2] = np.nan
    else:
        v = float("inf")
    setattr(b, field, v)
    dem, geo, init = _dropin_files(tmp_path, b)
    fd_dem, fd_geo = os.open(dem, os.O_RDONLY), os.open(geo, os.O_RDWR)
    try:
        with pytest.raises(_lib.SrgError) as e:
            api.azimuth_compress_status(b, fd_geo, fd_dem)
    finally:
        os.close(fd_dem)
        os.close(fd_geo)
    assert e.value.code == _lib.SRG_E_ARG
    assert f"non-finite value in {where}" in str(e.value)
    assert np.array_equal(np.fromfile(geo, np.complex64).reshape(init.shape), init)


def test_dropin_refuses_an_empty_box_and_a_scratch_limit(tmp_path):
    """latlons whose minimum latitude lies north of their maximum select no
    grid line (SRG_E_ARG); a scratch limit below the call's device scratch is
    SRG_E_NOMEM.  Both before any GPU work, the .geo untouched."""
    b = scene.mini_fixture(seed=11)
    dem, geo, init = _dropin_files(tmp_path, b)
    fd_dem, fd_geo = os.open(dem, os.O_RDONLY), os.open(geo, os.O_RDWR)
    try:
        inv = scene.mini_fixture(seed=11)
        inv.latlons = inv.latlons[[1, 0, 2, 3]].copy()
        with pytest.raises(_lib.SrgError) as e:
            api.azimuth_compress_status(inv, fd_geo, fd_dem)
        assert e.value.code == _lib.SRG_E_ARG and "no grid line" in str(e.value)
        with pytest.raises(_lib.SrgError) as e:
            api.azimuth_compress_status(b, fd_geo, fd_dem, scratch_limit=1 << 16)
        assert e.value.code == _lib.SRG_E_NOMEM and "limit" in str(e.value)
    finally:
        os.close(fd_dem)
        os.close(fd_geo)
    assert np.array_equal(np.fromfile(geo, np.complex64).reshape(init.shape), init)


def test_overlap_option_and_flush_without_a_gpu(monkeypatch):
    """The overlap option defaults off (SRG_DROPIN_OVERLAP unset), its field is
    where the header puts it, and a flush with no overlapped call made waits
    for nothing and succeeds on a machine without a GPU."""
    o = _lib.default_options()
    assert o.overlap == int(os.environ.get("SRG_DROPIN_OVERLAP", "0") == "1")
    assert _lib.Options.overlap.offset == _lib.Options.scratch_limit.offset + 8
    # the tile shear follows it and defaults to rectangular tiles
    assert _lib.Options.tile_shear.offset == _lib.Options.overlap.offset + 4
    assert o.tile_shear == 0
    assert _lib.lib().srg_dropin_flush(-1) == _lib.SRG_OK
    api.dropin_flush()


def test_overlap_environment_switch_sets_the_default():
    """SRG_DROPIN_OVERLAP=1 in the environment makes overlapped drop-in calls
    the process-wide default (srg_bp_default_options); other values do not."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); from srg_b200 import _lib; "
            "print(_lib.default_options().overlap)" % ROOT)
    for val, want in (("1", "1"), ("0", "0"), ("yes", "0")):
        env = dict(os.environ, SRG_DROPIN_OVERLAP=val)
        p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                           timeout=120)
        assert p.returncode == 0, p.stderr[-1000:]
        assert p.stdout.strip() == want, (val, p.stdout)


def _host_desc(b):
    """A descriptor with the burst's scalars only (no device memory): enough
    for srg_tile_shear, which reads nothing else."""
    fl, ll, fp, lp = api.limits(b)
    d = _lib.BurstDesc()
    d.P, d.S, d.demwidth = b.rawdatalines, b.samples, b.demwidth
    d.firstline, d.nlines, d.firstpix, d.lastpix = fl, ll - fl + 1, fp, lp
    d.aperture = b.aperture
    d.firstlat, d.deltalat, d.firstlon, d.deltalon = b.firstlat, b.deltalat, b.firstlon, b.deltalon
    d.rngstart, d.rngend, d.dmrg, d.wvl = b.rngstart, b.rngend, b.dmrg, b.wvl
    for i in range(3):
        d.xyz_mid[i] = float(b.xyz_mid[i])
        d.vel_mid[i] = float(b.vel_mid[i])
    d.prf = b.prf
    return d


def _shear(d, cfg=-1, forced=_lib.TILE_SHEAR_AUTO):
    s, tx, ty = C.c_int(), C.c_int(), C.c_int()
    rc = _lib.lib().srg_tile_shear(C.byref(d), cfg, forced, C.byref(s), C.byref(tx), C.byref(ty))
    return rc, s.value, tx.value, ty.value


def test_tile_shear_follows_the_azimuth_centres():
    """On the IW scene the azimuth centre moves ~2.43 pulses per grid line
    and ~0.56 per column, the range ~0.6-1.0 bins per line and ~2.5-3.0 per
    column.  The default 32 x 8 tiles shear by -7 lines per 32 columns: each
    tile's rows of pixels then follow the lines of constant centre (measured
    with the oracle's windows: 3.6 % fewer pixel-pulse slots, 7.6 % fewer
    chunks) and widen its range window by ~4 bins; a column then needs
    ceil((nlines + 7) / 8) tiles.  First-generation shapes keep rectangular
    tiles; a forced shear is taken as given and one out of range, or one that
    offsets a tile's columns by its height or more, is refused."""
    _, bursts = scene.iw_scene(seed=1003)
    first_gen = [c[0] for c in _lib.tile_configs() if "bp_tiles" in _lib.tile_config_name(c[0])]
    assert first_gen
    for b in bursts[:3]:
        d = _host_desc(b)
        nx = min(d.lastpix, d.demwidth - 1) - d.firstpix + 1
        rc, s, tx, ty = _shear(d)
        assert rc == _lib.SRG_OK and s == -7, (rc, s)
        assert tx == -(-nx // 32) and ty == -(-(d.nlines + 7) // 8)
        assert all(_shear(d, cfg)[1] == 0 for cfg in first_gen)
        assert _shear(d, -1, 3)[:2] == (_lib.SRG_OK, 3)
        assert _shear(d, -1, 0)[1:] == (0, -(-nx // 32), -(-d.nlines // 8))
        assert _shear(d, -1, 9)[0] == _lib.SRG_E_ARG
        assert _shear(d, -1, 8)[0] == _lib.SRG_OK     # offset floor(8 * 31 / 32) = 7 < 8
    # without a velocity (a caller passing its own centres) the tiles stay rectangular
    d = _host_desc(bursts[0])
    for i in range(3):
        d.vel_mid[i] = 0.0
    assert _shear(d)[1] == 0
