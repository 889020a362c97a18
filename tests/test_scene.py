"""Synthetic scene generator: orbit interpolation accuracy and the derived
burst parameters."""
import numpy as np

from srg_b200 import scene


def test_hermite_matches_analytic_orbit():
    b = scene.make_geometry(pulses=1500, samples=21000, width=64, length=64, spacing=1e-4,
                            quantise=False)
    orb = scene.CircularOrbit(u0=np.arcsin(np.sin(np.radians(19.4)) / np.sin(np.radians(98.18))),
                              epoch=43200.25)
    x, v = orb.state(b.pulse_time)
    assert np.max(np.linalg.norm(b.satloc - x, axis=1)) < 1e-3       # < 1 mm
    assert np.max(np.linalg.norm(b.satvel - v, axis=1)) < 1e-5


def test_config_aperture_and_spacing():
    b = scene.make_geometry(pulses=1500, samples=21000, width=64, length=64, spacing=1e-4)
    assert abs(b.dmrg - 2.3295) < 1e-3
    # ~700 pulses: r = 7071 km (|v| ~ 7.4 km/s in the rotating frame), near range 800 km
    assert 680 <= b.aperture <= 730
    assert b.numstatevec == 11 and np.allclose(np.diff(b.timeorbit), 10.0)


def test_mini_samples_are_reproducible():
    a = scene.mini_samples(5, 16, 32)
    c = scene.mini_samples(5, 16, 32)
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
    assert np.all(np.abs(a.real * 16 - np.rint(a.real * 16)) == 0)


def test_text_quantisation_round_trip():
    x = np.array([[7071000.123456789, -1.5, 2.25]])
    v = np.array([[7500.123456789, 0.0, -3.0]])
    xq, vq = scene.quantise_positions(x, v)
    assert xq[0, 0] == 7071000.1234568 and vq[0, 0] == 7500.12345679
