"""Failure detection, tested without a GPU fault: device-side waits that run
out (a word nothing raises, a poll limit shorter than the upload), host-side
injections (a truncated DEM file, a grid box outside the DEM), and the
drop-in's call number restarting.  Every failure must come back as a status,
with nothing half-merged into the .geo raster."""
import ctypes as C
import os
import tempfile
import time

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


def gated(torch, db, word, base, rows, spin=0):
    o = _lib.default_options(_lib.FORM_SPLIT)
    o.spin_limit = spin
    d = db.desc()
    st = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib().srg_bp_burst_device_gated(C.byref(d), C.c_void_p(word.data_ptr()), base, rows,
                                              C.byref(o), C.c_void_p(st))
    assert rc == _lib.SRG_OK, _lib.last_error()
    return _lib.lib().srg_sync_check(C.c_void_p(st))


def test_gated_burst_equals_the_plain_entry_when_the_lines_are_in(torch_cuda):
    torch = torch_cuda
    b = mini_case("tops")
    db = api.to_device(b)
    api.backproject([db], form=_lib.FORM_SPLIT)
    ref = db.out.clone()
    rows = 10
    word = torch.full((1,), 64 + (b.rawdatalines + rows - 1) // rows, dtype=torch.int32,
                      device="cuda")
    db.out.fill_(complex(5.0, 5.0))
    assert gated(torch, db, word, 64, rows) == _lib.SRG_OK
    assert torch.equal(db.out.view(torch.float32), ref.view(torch.float32))


def test_gated_wait_that_runs_out_returns_timeout(torch_cuda):
    """The upload word is never raised: every CTA's wait gives up after the
    short poll limit, the call returns SRG_E_TIMEOUT within a second, no tile
    is stored, and the context stays usable (the next call is exact)."""
    torch = torch_cuda
    b = mini_case("tops")
    db = api.to_device(b)
    api.backproject([db], form=_lib.FORM_SPLIT)
    ref = db.out.clone()
    word = torch.zeros((1,), dtype=torch.int32, device="cuda")
    db.out.fill_(complex(5.0, 5.0))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = gated(torch, db, word, 64, 10, spin=256)
    dt = time.perf_counter() - t0
    assert rc == _lib.SRG_E_TIMEOUT, _lib.last_error()
    assert dt < 1.0, dt
    # tiles that never got their lines keep the old output
    out = db.out.cpu().numpy()
    assert np.count_nonzero(out == np.complex64(5 + 5j)) > 0
    assert not np.any((out != np.complex64(5 + 5j)) & (out != 0))
    # the error word is cleared and the context works
    assert _lib.lib().srg_sync_check(C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    db.out.zero_()
    api.backproject([db], form=_lib.FORM_SPLIT)
    assert torch.equal(db.out.view(torch.float32), ref.view(torch.float32))


def _run_dropin(b, geo_init, host_lines, dem=None, **options):
    """One status call of the drop-in on temp files; (rc, resulting .geo)."""
    with tempfile.TemporaryDirectory() as td:
        dem_path, geo_path = os.path.join(td, "e.dem"), os.path.join(td, "s.geo")
        np.ascontiguousarray(b.dem if dem is None else dem, np.int16).tofile(dem_path)
        np.ascontiguousarray(geo_init, np.complex64).tofile(geo_path)
        fd_dem, fd_geo = os.open(dem_path, os.O_RDWR), os.open(geo_path, os.O_RDWR)
        try:
            try:
                api.azimuth_compress_status(b, fd_geo, fd_dem, burst=host_lines, **options)
                rc = _lib.SRG_OK
            except _lib.SrgError as e:
                rc = e.code
        finally:
            os.close(fd_dem)
            os.close(fd_geo)
        return rc, np.fromfile(geo_path, np.complex64).reshape(geo_init.shape)


def test_dropin_wait_that_gives_up_merges_only_whole_rows(torch_cuda):
    """Pinned range lines upload in blocks while the kernel runs; with a poll
    limit far shorter than the upload the kernel gives up on chunks whose rows
    are not in yet.  The call returns SRG_E_TIMEOUT and every .geo row is
    either as it was or exactly the row a complete call writes: a row block is
    merged only when every one of its kept tiles was stored."""
    torch = torch_cuda
    b = scene.config0_point_targets()
    rng = np.random.default_rng(3)
    init = (rng.standard_normal((b.demlength, b.demwidth)) +
            1j * rng.standard_normal((b.demlength, b.demwidth))).astype(np.complex64)
    pinned = torch.from_numpy(np.ascontiguousarray(b.burst, np.complex64)).pin_memory()
    rc, full = _run_dropin(b, init, pinned.numpy())
    assert rc == _lib.SRG_OK
    changed = full != init
    assert changed.any()
    timeouts = 0
    for _ in range(3):
        rc, got = _run_dropin(b, init, pinned.numpy(), spin_limit=8)
        assert rc in (_lib.SRG_OK, _lib.SRG_E_TIMEOUT)
        timeouts += rc == _lib.SRG_E_TIMEOUT
        for r in range(b.demlength):
            assert (np.array_equal(got[r].view(np.uint32), init[r].view(np.uint32)) or
                    np.array_equal(got[r].view(np.uint32), full[r].view(np.uint32))), r
        if rc == _lib.SRG_OK:
            assert np.array_equal(got.view(np.uint32), full.view(np.uint32))
    assert timeouts > 0
    # and a call with the default limit is complete again
    rc, again = _run_dropin(b, init, pinned.numpy())
    assert rc == _lib.SRG_OK and np.array_equal(again.view(np.uint32), full.view(np.uint32))


def test_dropin_truncated_dem_is_an_error(torch_cuda):
    b = mini_case("slope")
    init = np.full((b.demlength, b.demwidth), 1 + 2j, np.complex64)
    fl, ll, _, _ = api.limits(b)
    short = np.ascontiguousarray(b.dem, np.int16)[:(fl + ll) // 2]  # ends inside the box
    rc, got = _run_dropin(b, init, b.burst, dem=short)
    assert rc == _lib.SRG_E_IO
    assert "ends before" in _lib.last_error()
    assert np.array_equal(got, init)


def test_dropin_box_outside_the_dem_forms_nothing(torch_cuda):
    """A lat/lon box north of the DEM clamps to its first line (one line,
    which the reference never forms): OK, the .geo untouched."""
    b = mini_case("slope")
    b.latlons = b.latlons.copy()
    b.latlons[:2] = b.firstlat + np.array([5.0, 6.0]) * abs(b.deltalat) * b.demlength
    init = np.full((b.demlength, b.demwidth), 1 + 2j, np.complex64)
    rc, got = _run_dropin(b, init, b.burst)
    assert rc == _lib.SRG_OK
    assert np.array_equal(got, init)


def test_dropin_call_number_restart(torch_cuda):
    """The drop-in tells a call's uploaded rows from an earlier call's by a
    call number in a device word; across its restart (after 2^24 calls) the
    words are cleared first.  Two bursts with different lines alternate
    across the restart: every .geo equals the one a fresh call writes."""
    torch = torch_cuda
    a = scene.config0_point_targets(seed=1000)
    c = scene.config0_point_targets(seed=1001)
    c.dem = a.dem
    zero = np.zeros((a.demlength, a.demwidth), np.complex64)
    hosts = [torch.from_numpy(np.ascontiguousarray(x.burst, np.complex64)).pin_memory().numpy()
             for x in (a, c)]
    refs = [_run_dropin(x, zero, h)[1] for x, h in zip((a, c), hosts)]
    assert not np.array_equal(refs[0], refs[1])
    L = _lib.lib()
    assert L.srg_test_set_dropin_sequence(-1, (1 << 24) - 2) == _lib.SRG_OK
    try:
        for i in range(6):
            k = i % 2
            rc, got = _run_dropin((a, c)[k], zero, hosts[k])
            assert rc == _lib.SRG_OK
            assert np.array_equal(got.view(np.uint32), refs[k].view(np.uint32)), i
    finally:
        L.srg_test_set_dropin_sequence(-1, 0)
