"""The oracle (CPU restatement) against the golden fixtures made by the
compiled reference, and against the compiled reference itself when it is
present (oracle/_ref)."""
import os

import numpy as np
import pytest

import oracle as O
from helpers import MINI_CASES, load_golden, mini_case, rel_err
from srg_b200 import scene

NAMES = [c[0] for c in MINI_CASES]


@pytest.fixture(scope="module")
def orc():
    O.build()
    return O.Oracle()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(orc, name):
    b, g = load_golden(name)
    st = orc.stages(b, gpu_lerp=0, gpu_scale=0)
    fl, ll, fp, lp = (int(v) for v in g["limits"])
    assert (st["firstline"], st["firstline"] + st["nlines"] - 1, st["firstpix"], st["lastpix"]) == (fl, ll, fp, lp)
    # ECEF: libm sin/cos may differ by an ulp between hosts (1e-9 m here)
    np.testing.assert_allclose(st["xyz"], g["ref_xyz"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(st["xyzfit"], g["ref_xyzfit"], rtol=0, atol=1e-7)
    # aperture centres are integer arithmetic: exact
    assert np.array_equal(st["azoff"], g["ref_azoff"])
    assert st["terms"] == int(g["terms"])
    # raw sums on the reference's own ECEF/azoff inputs
    out, _, terms = orc.pixelint(b, g["ref_xyz"], g["ref_azoff"], gpu_lerp=0, gpu_scale=0)
    assert terms == int(g["terms"])
    assert rel_err(out, g["ref_pixelint"]) < 1e-6
    # end to end, CPU merge rule; the last burst line is excluded (the
    # reference reads a parabola it never computed there)
    geo, _ = orc.burst_geo(b, gpu=False)
    ref = g["ref_geo"]
    keep = np.ones(ref.shape[0], bool)
    keep[ll] = False
    assert np.array_equal(geo[keep] != 0, ref[keep] != 0)
    assert rel_err(geo[keep], ref[keep]) < 1e-6


@pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="compiled reference not built here")
@pytest.mark.parametrize("name", NAMES)
def test_restatement_bitexact_vs_compiled_reference(orc, name):
    b = mini_case(name)
    r = O.RefCPU()
    st = orc.stages(b, gpu_lerp=0, gpu_scale=0)
    xyz, fit = r.setxyz(b, st["firstline"], st["nlines"], st["firstpix"], st["lastpix"])
    assert np.array_equal(xyz, st["xyz"]) and np.array_equal(fit, st["xyzfit"])
    az = r.setazoff(b, st["coef"], st["firstpix"], st["lastpix"])
    assert np.array_equal(az, st["azoff"])
    pix = r.pixelint(b, st["xyz"], st["azoff"])
    assert np.array_equal(pix.view(np.uint32), st["out"].view(np.uint32))
    geo_ref = r.azimuth_compress_cpu(b)
    geo, _ = orc.burst_geo(b, gpu=False)
    last = st["firstline"] + st["nlines"] - 1
    keep = np.ones(geo.shape[0], bool)
    keep[last] = False
    assert np.array_equal(geo[keep].view(np.uint32), geo_ref[keep].view(np.uint32))


def test_gpu_form_of_oracle_scales_and_lerps(orc):
    """GPU-form variant: FP32 lerp + 1/(azend-azstart) scaling
    (azimuth_compress.cu:69, 78-79); differs from the CPU form only by them."""
    b = mini_case("slope")
    st_c = orc.stages(b, gpu_lerp=0, gpu_scale=0)
    st_g = orc.stages(b, gpu_lerp=1, gpu_scale=1)
    az = st_c["azoff"]
    a0 = np.round(az - b.aperture // 2).astype(int)
    a1 = np.round(az + b.aperture // 2).astype(int)
    n = np.clip(a1, None, b.rawdatalines - 1) - np.clip(a0, 0, None)
    formed = az > 0
    scaled = st_c["out"][formed] * (1.0 / n[formed]).astype(np.float32)
    assert rel_err(st_g["out"][formed], scaled) < 1e-5
    assert np.all(st_g["out"][~formed] == 0)


def test_orbit_helpers(orc):
    """Hermite restatement vs the scene generator's own Hermite, the clamp of
    intp_orbit, and the zero-Doppler condition of orbitrangetime."""
    import ctypes as C
    b = mini_case("flat")
    L = orc.lib
    dp = C.POINTER(C.c_double)
    to = np.ascontiguousarray(b.timeorbit)
    xx = np.ascontiguousarray(b.xx)
    vv = np.ascontiguousarray(b.vv)
    n = C.c_int(len(to))
    for t in (b.tstart, b.tmid, b.tend, to[0] - 5.0, to[-1] + 3.0):
        x = np.zeros(3)
        v = np.zeros(3)
        L.intp_orbit_(to.ctypes.data_as(dp), xx.ctypes.data_as(dp), vv.ctypes.data_as(dp),
                      C.byref(n), C.byref(C.c_double(t)), x.ctypes.data_as(dp), v.ctypes.data_as(dp))
        xs, vs = scene.intp_orbit(to, xx, vv, t)
        np.testing.assert_allclose(x, xs, rtol=0, atol=1e-6)
        np.testing.assert_allclose(v, vs, rtol=0, atol=1e-9)
    # a ground point: Newton lands on zero Doppler
    g = scene.grid_ecef(b, 20, 24, 200.0)
    tl, rg = C.c_double(), C.c_double()
    L.orbitrangetime_(g.ctypes.data_as(dp), to.ctypes.data_as(dp), xx.ctypes.data_as(dp),
                      vv.ctypes.data_as(dp), C.byref(n), C.byref(C.c_double(b.tmid)),
                      np.ascontiguousarray(b.xyz_mid).ctypes.data_as(dp),
                      np.ascontiguousarray(b.vel_mid).ctypes.data_as(dp), C.byref(tl), C.byref(rg))
    xs, vs = scene.intp_orbit(to, xx, vv, tl.value)
    d = g - xs
    assert abs(np.dot(d, vs)) / (np.linalg.norm(d) * np.linalg.norm(vs)) < 1e-9
    assert abs(np.linalg.norm(d) - rg.value) < 1e-6
