"""The drop-in uploads only the range band of each burst: the range bins a
term of a formed pixel can read (found on the device from the DEM box and
the azimuth centres, with a margin), instead of every line in full as the
reference does (sentinel/azimuth_compress.cu:367-368).  The .geo it writes
must be bit-identical to the full-line upload's, in both forms, on the mini
cases and on the IW1-sized burst, with far fewer bytes copied in."""
import os
import tempfile

import numpy as np
import pytest

from helpers import mini_case
from srg_b200 import _lib, api, scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def dropin(b, init, lines, form, full_lines):
    with tempfile.TemporaryDirectory() as td:
        dem_path, geo_path = os.path.join(td, "e.dem"), os.path.join(td, "s.geo")
        np.ascontiguousarray(b.dem, np.int16).tofile(dem_path)
        np.ascontiguousarray(init, np.complex64).tofile(geo_path)
        fd_dem, fd_geo = os.open(dem_path, os.O_RDWR), os.open(geo_path, os.O_RDWR)
        try:
            api.azimuth_compress_status(b, fd_geo, fd_dem, form=form, burst=lines,
                                        full_lines=full_lines)
            h2d, d2h = api.dropin_last_bytes()
        finally:
            os.close(fd_dem)
            os.close(fd_geo)
        return np.fromfile(geo_path, np.complex64).reshape(init.shape), h2d, d2h


def check(b, lines, form):
    rng = np.random.default_rng(9)
    init = (rng.standard_normal((b.demlength, b.demwidth)) +
            1j * rng.standard_normal((b.demlength, b.demwidth))).astype(np.complex64)
    full, h_full, _ = dropin(b, init, lines, form, 1)
    band, h_band, _ = dropin(b, init, lines, form, 0)
    assert (full != init).sum() > 0
    assert np.array_equal(band.view(np.uint32), full.view(np.uint32))
    assert h_band <= h_full
    return h_band, h_full


@pytest.mark.parametrize("form", [_lib.FORM_SPLIT, _lib.FORM_FP64])
@pytest.mark.parametrize("name", ["slope", "inset", "oddS", "tops"])
def test_band_upload_bit_identical_mini(torch_cuda, name, form):
    b = mini_case(name)
    check(b, b.burst, form)


@pytest.mark.parametrize("form", [_lib.FORM_SPLIT, _lib.FORM_FP64])
def test_band_upload_bit_identical_point_targets(torch_cuda, form):
    """Configuration 0 from pinned lines (the pipelined upload with the
    split form's gated kernel)."""
    torch = torch_cuda
    b = scene.config0_point_targets()
    pinned = torch.from_numpy(np.ascontiguousarray(b.burst, np.complex64)).pin_memory()
    check(b, pinned.numpy(), form)


@pytest.mark.parametrize("form", [_lib.FORM_SPLIT, _lib.FORM_FP64])
def test_band_upload_bit_identical_iw1_burst(torch_cuda, form):
    """The IW1-sized burst (1,500 x 21,000 forward-projected lines, 2,400 x
    1,200 grid over the volcano DEM): same .geo, and the band is a fraction of
    the lines (the grid's slant-range extent is a third of the swath)."""
    torch = torch_cuda
    from srg_b200 import workloads
    wl = workloads.config1()
    db = wl.bursts[0]
    pinned = torch.empty(tuple(db.burst.shape), dtype=torch.complex64, pin_memory=True)
    pinned.copy_(db.burst)
    h_band, h_full = check(db.b, pinned.numpy(), form)
    assert h_band < 0.6 * h_full, (h_band, h_full)
