"""The C ABI library without a GPU: it loads, exports every entry point that
include/srg_bp.h declares, and reports its kernel shapes.  No compute call."""
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
