"""Per-burst scalars of the azimuth_compress_ call (srg_burst_params, host
code of libsrg_bp.so) against the oracle's restatement of
sentinel/backprojectgpusub.f90's burstparams, fdopcoefs, aperture and limits
(oracle/params.py), on synthetic Sentinel-1 line headers.  No GPU needed."""
import numpy as np
import pytest

import params as OP
from srg_b200 import _lib, api, build, scene

FIELDS = ("starttime", "prf", "samplefreq", "pri", "range0", "wvl", "angc0", "angc1", "tstart",
          "tend", "tmid", "dtaz", "rngstart", "rngend", "dmrg", "aperture")


@pytest.fixture(scope="module", autouse=True)
def built():
    build.build()


def lines_with_headers(P, S, seed, decimation=8, rank=9, steer=(-0.7, 0.7), jitter=0):
    """Decoded lines of one burst: random samples, the first 10 of each line
    holding its header (line times at the PRF, a linear TOPS steering sweep of
    the azimuth beam address with optional +-jitter address noise)."""
    rng = np.random.default_rng(seed)
    b = scene.make_geometry(pulses=P, samples=S, width=8, length=8, spacing=1e-4, quantise=False)
    pri_code, swst_code = scene.header_codes(b.prf, b.rngstart, rank)
    ang = np.linspace(steer[0], steer[1], P)
    addr = np.clip(np.rint((ang + 0.9) / 1.8 * 1024).astype(np.int64) +
                   (rng.integers(-jitter, jitter + 1, P) if jitter else 0), 0, 1023)
    lines = (rng.standard_normal((P, S)) + 1j * rng.standard_normal((P, S))).astype(np.complex64)
    lines[:, :10] = scene.encode_line_headers(b.pulse_time, pri_code, rank, swst_code, decimation,
                                              addr)
    return b, lines


def oracle_params(lines, satvel):
    hdr = np.ascontiguousarray(lines[:, :10]).view(np.uint8).reshape(lines.shape[0], 80)
    return OP.burst_params(hdr, satvel, lines.shape[1])


@pytest.mark.parametrize("case", [
    dict(P=1500, S=600, seed=1),
    dict(P=1451, S=333, seed=2, decimation=1, rank=10, steer=(-0.6, 0.8), jitter=3),
    dict(P=41, S=11, seed=3, decimation=0, steer=(0.3, -0.2)),
    dict(P=2001, S=64, seed=4, decimation=11, jitter=40),
])
def test_burst_params_match_the_oracle_bit_for_bit(case):
    P, S, seed = case.pop("P"), case.pop("S"), case.pop("seed")
    b, lines = lines_with_headers(P, S, seed, **case)
    got = api.burst_params(lines, b.satvel)
    want = oracle_params(lines, b.satvel)
    for k in FIELDS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_burst_params_decode_the_synthetic_radar():
    """The decoded values are those the headers were made from (PRF and
    near range to the codes' rounding, 64.345 MHz for decimation code 8, the
    wavelength literal, a positive steering rate for a forward sweep) and
    the aperture follows the TOPS formula of the synthetic scenes."""
    b, lines = lines_with_headers(1500, 600, 7)
    p = api.burst_params(lines, b.satvel)
    assert abs(p["prf"] - scene.PRF) < 0.05
    assert abs(p["range0"] - b.rngstart) < 2.0
    assert abs(p["samplefreq"] - 64.345e6) < 1e3
    assert p["wvl"] == float(np.float32(0.05546576))
    assert p["angc1"] > 1.0 and abs(p["angc0"]) < 0.01          # deg/s, deg
    assert p["aperture"] == scene.aperture_points(b.satvel, p["range0"], p["wvl"], p["prf"],
                                                  p["angc1"])
    assert p["tmid"] == 0.5 * (p["tstart"] + p["tend"])
    assert p["rngend"] == p["rngstart"] + (lines.shape[1] - 1) * p["dmrg"]


def test_burst_params_reject_bad_headers():
    b, lines = lines_with_headers(100, 64, 8)
    with pytest.raises(_lib.SrgError) as e:
        api.burst_params(lines[:40], b.satvel[:40])       # needs 41 lines
    assert e.value.code == _lib.SRG_E_ARG
    bad = lines.copy()
    bad[:, :10] = scene.encode_line_headers(b.pulse_time, 21859, 9, 100, 2, 512)  # code 2: none
    with pytest.raises(_lib.SrgError) as e:
        api.burst_params(bad, b.satvel)
    assert "decimation" in str(e.value)
