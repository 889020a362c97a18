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
