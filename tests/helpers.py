"""Shared helpers of the test suite: scenes, fixtures and error metrics."""
from __future__ import annotations

import os

import numpy as np

from srg_b200 import scene

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

# The mini scenes of the golden fixtures: (name, kwargs of scene.mini_fixture).
MINI_CASES = [
    ("flat", dict(seed=11, dem_kind="flat")),
    ("slope", dict(seed=12, dem_kind="slope")),
    ("tops", dict(seed=13, dem_kind="slope", angc0=0.05, angc1=0.4)),
    ("inset", dict(seed=14, dem_kind="slope", latlons_inset=5)),
    ("oddS", dict(seed=15, dem_kind="slope", samples=383, pulses=300, aperture=80)),
]


def mini_case(name: str) -> scene.Burst:
    kw = dict(MINI_CASES)[name]
    return scene.mini_fixture(**kw)


def load_golden(name: str):
    """(Burst rebuilt from the fixture, dict of stored reference outputs)."""
    path = os.path.join(GOLDEN, f"mini_{name}.npz")
    z = np.load(path)
    P, S = [int(v) for v in z["ints"][-2:]]
    b = scene.burst_from_arrays(z, scene.mini_samples(int(z["sample_seed"]), P, S))
    return b, {k: z[k] for k in z.files}


def phase_amp_errors(test: np.ndarray, ref: np.ndarray, floor_frac: float = 0.05):
    """Phase error (mrad: RMS, max) and amplitude relative error (RMS, max)
    over pixels whose reference amplitude exceeds floor_frac x RMS amplitude."""
    test = np.asarray(test, np.complex128).ravel()
    ref = np.asarray(ref, np.complex128).ravel()
    amp = np.abs(ref)
    nz = amp > 0
    if not np.any(nz):
        return dict(n=0, ph_rms=0.0, ph_max=0.0, amp_rms=0.0, amp_max=0.0)
    floor = floor_frac * np.sqrt(np.mean(amp[nz] ** 2))
    m = amp > floor
    ph = np.angle(test[m] * np.conj(ref[m])) * 1e3
    ar = np.abs(np.abs(test[m]) - amp[m]) / amp[m]
    return dict(n=int(m.sum()), ph_rms=float(np.sqrt(np.mean(ph ** 2))),
                ph_max=float(np.max(np.abs(ph))), amp_rms=float(np.sqrt(np.mean(ar ** 2))),
                amp_max=float(np.max(ar)))


def rel_err(test, ref, floor_frac=1e-3):
    """max |test - ref| / max(|ref|, floor) with floor = floor_frac * max|ref|."""
    test = np.asarray(test, np.complex128)
    ref = np.asarray(ref, np.complex128)
    floor = max(floor_frac * np.abs(ref).max(), 1e-30)
    return float(np.max(np.abs(test - ref) / np.maximum(np.abs(ref), floor)))
