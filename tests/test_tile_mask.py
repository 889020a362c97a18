"""The work list's tile test (kernels.cu: tile_mask_kernel), restated in numpy:
a tile is dropped only when every one of its lines' azimuth-centre parabolas
stays outside (ap2, P - ap2) over the tile's columns on that line (ends and
vertex, margin 1e-3 pulse; a sheared tile's columns sit on lines offset by
floor(shear x / 32), so each line holds one interval of them).  Checked on
CPU against the oracle's per-pixel azoff: the tiles partition the grid, no
dropped tile may hold a formed pixel, and on grids that reach past the
pulses most tiles without one are dropped.  (The GPU tests check the
kernel's outputs.)"""
import math

import numpy as np
import pytest

import oracle as O
from helpers import MINI_CASES, mini_case
from srg_b200 import scene


def _fit(c, a):
    return (c[0] * a) * a + c[1] * a + c[2]


def dline(shear, x):
    """Line offset of a tile's column x (common.cuh: tile_dline):
    floor(shear * x / 32)."""
    return (shear * x) // 32


def tile_lines(ty_row, x, tx, ty, shear):
    """Lines of tile row ty_row on its column x (common.cuh: the tile geometry)."""
    dmax = dline(shear, tx - 1) if shear > 0 else 0
    l0 = ty_row * ty + dline(shear, x) - dmax
    return l0, l0 + ty


def tile_keep(coef, fp, lp, lastpix_eff, nlines, ap2, P, tx, ty, shear=0):
    den = np.float32(lp - fp)
    span = abs(dline(shear, tx - 1))
    ntx = math.ceil((lastpix_eff - fp + 1) / tx)
    nty = math.ceil((nlines + span) / ty)
    keep = np.zeros((nty, ntx), bool)
    for ti in range(nty):
        for tj in range(ntx):
            k = False
            for line in range(ti * ty - span, ti * ty + ty):
                if not 0 <= line < nlines:
                    continue
                xs = [x for x in range(tx) if tile_lines(ti, x, tx, ty, shear)[0] <= line <
                      tile_lines(ti, x, tx, ty, shear)[1]]
                if not xs:
                    continue
                px0, px1 = fp + tj * tx + xs[0], min(fp + tj * tx + xs[-1], lastpix_eff)
                if px0 > px1:
                    continue
                assert xs == list(range(xs[0], xs[-1] + 1))   # one interval per line
                a0 = float(np.float32(np.float32(px0 - fp) / den)) * 2.0 - 1.0
                a1 = float(np.float32(np.float32(px1 - fp) / den)) * 2.0 - 1.0
                c = coef[line]
                f0, f1 = _fit(c, a0), _fit(c, a1)
                lo, hi = min(f0, f1), max(f0, f1)
                if c[0] != 0.0:
                    v = -c[1] / (2.0 * c[0])
                    if a0 < v < a1:
                        fv = _fit(c, v)
                        lo, hi = min(lo, fv), max(hi, fv)
                if not all(np.isfinite([f0, f1, lo, hi])):
                    k = True
                elif not (hi < ap2 - 1e-3 or lo > P - ap2 + 1e-3):
                    k = True
            keep[ti, tj] = k
    return keep


def formed(azoff, ap2, P):
    """aze > azs of every pixel (the kernel's pixel_window)."""
    ok = azoff > 0.0
    azs = np.maximum(np.round(azoff - ap2), 0)
    aze = np.minimum(np.round(azoff + ap2), P - 1)
    return ok & (aze > azs)


CASES = [c[0] for c in MINI_CASES] + ["long", "long_tops"]


def _burst(name):
    if name == "long":
        return scene.mini_fixture(seed=31, length=400, width=96)
    if name == "long_tops":
        return scene.mini_fixture(seed=32, length=300, width=80, angc0=0.05, angc1=0.4)
    return mini_case(name)


@pytest.fixture(scope="module")
def orc():
    O.build()
    return O.Oracle()


@pytest.mark.parametrize("tx,ty,shear", [(32, 8, 0), (8, 4, 0), (16, 16, 0), (32, 8, -7),
                                          (32, 8, 3), (16, 16, -8), (32, 4, 4)])
@pytest.mark.parametrize("name", CASES)
def test_dropped_tiles_hold_no_formed_pixel(orc, name, tx, ty, shear):
    b = _burst(name)
    st = orc.stages(b)
    fp, lp, nl = st["firstpix"], st["lastpix"], st["nlines"]
    lpe = min(lp, b.demwidth - 1)
    ap2, P = b.aperture // 2, b.rawdatalines
    keep = tile_keep(st["coef"], fp, lp, lpe, nl, ap2, P, tx, ty, shear)
    f = formed(st["azoff"][:, fp:lpe + 1], ap2, P)
    has = np.zeros_like(keep)
    covered = np.zeros_like(f, dtype=np.int32)
    for ti in range(keep.shape[0]):
        for tj in range(keep.shape[1]):
            for x in range(tx):
                c = tj * tx + x
                if c >= f.shape[1]:
                    continue
                l0, l1 = tile_lines(ti, x, tx, ty, shear)
                l0, l1 = max(l0, 0), min(l1, nl)
                if l0 < l1:
                    has[ti, tj] |= f[l0:l1, c].any()
                    covered[l0:l1, c] += 1
    assert np.all(covered == 1)              # the tiles partition the grid
    assert not np.any(has & ~keep)          # safety: nothing formed is dropped
    if name.startswith("long"):              # and the empty tiles mostly go
        empty = ~has
        assert empty.sum() > 0.5 * has.size
        assert (empty & ~keep).sum() >= 0.9 * empty.sum()
