"""srg_bp_burst_device_noalloc: the entry point for callers that cannot call
cudaMalloc (a process whose device memory is held by a pool it does not
own, or a latency-critical stream that cannot take cudaMalloc/cudaFree's
device-wide synchronisation).  Its scratch is a static device array shared
by every call, so the test calls it on several bursts back to back and
checks each result against the allocating entry (srg_bp_bursts_device).

Kept in its own file, collected last, so that a failure here stops a `-x`
run only after every other test has run; it also passes alone in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import mini_case, rel_err
from srg_b200 import _lib, api

pytestmark = pytest.mark.gpu

# Same tolerance as the FP64-form parity tests (the two entries run the same
# kernel on the same inputs, so the outputs are expected to be identical).
REL_TOL = 2e-6


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the CUDA path needs a GPU; none is visible")
    return torch


def call_noalloc(torch, db, form):
    o = _lib.default_options(form)
    d = db.desc()
    st = torch.cuda.current_stream().cuda_stream
    return _lib.lib().srg_bp_burst_device_noalloc(C.byref(d), C.byref(o), C.c_void_p(st))


@pytest.mark.parametrize("form", [_lib.FORM_SPLIT, _lib.FORM_FP64])
def test_noalloc_matches_allocating_entry_on_consecutive_calls(torch_cuda, form):
    torch = torch_cuda
    # bursts of different sizes, called one after the other, then the first
    # one again: stale scratch from a previous call must not leak into a result
    names = ["tops", "oddS", "inset", "tops"]
    for name in names:
        b = mini_case(name)
        db = api.to_device(b)
        api.backproject([db], form=form)
        # both entries write the burst's pixel window [firstpix, min(lastpix, W-1)]
        win = slice(db.firstpix, min(db.lastpix, b.demwidth - 1) + 1)
        ref = db.out.cpu().numpy()[:, win]
        sentinel = complex(7.0, -7.0)
        for _ in range(2):
            db.out.fill_(sentinel)
            rc = call_noalloc(torch, db, form)
            assert rc == _lib.SRG_OK, _lib.last_error()
            full = db.out.cpu().numpy()
            got = full[:, win]
            assert np.array_equal(got != 0, ref != 0)
            assert rel_err(got, ref) < REL_TOL
            outside = np.ones(full.shape[1], bool)
            outside[win] = False
            assert np.all(full[:, outside] == sentinel)


def test_noalloc_allocates_nothing(torch_cuda):
    """After the first call on a device (which may load the kernels), calls
    leave the device's free memory exactly as they found it: nothing is
    allocated, by the library or by torch (the buffers exist before the
    calls, and the calls go through ctypes)."""
    torch = torch_cuda
    b = mini_case("tops")
    db = api.to_device(b)
    for form in (_lib.FORM_SPLIT, _lib.FORM_FP64):
        assert call_noalloc(torch, db, form) == _lib.SRG_OK, _lib.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for form in (_lib.FORM_SPLIT, _lib.FORM_FP64):
            assert call_noalloc(torch, db, form) == _lib.SRG_OK, _lib.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_refuses_host_centres_like_the_allocating_entry(torch_cuda):
    torch = torch_cuda
    b = mini_case("flat")
    db = api.to_device(b)
    o = _lib.default_options(_lib.FORM_SPLIT)
    o.centres_on_host = 1
    d = db.desc()
    st = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib().srg_bp_burst_device_noalloc(C.byref(d), C.byref(o), C.c_void_p(st))
    assert rc == _lib.SRG_E_UNSUPPORTED
    rc2 = _lib.lib().srg_bp_bursts_device(C.byref(d), 1, C.byref(o), C.c_void_p(st))
    assert rc2 == _lib.SRG_E_UNSUPPORTED


def test_noalloc_rejects_bursts_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    b = mini_case("flat")
    db = api.to_device(b)
    n = 8193  # SRG_NOALLOC_MAX_LINES + 1
    # buffers really hold n lines, so nothing could be read out of bounds
    # even if the check were missing
    db.dem = torch.zeros((n, b.demwidth), dtype=torch.int16, device="cuda")
    db.out = torch.zeros((n, b.demwidth), dtype=torch.complex64, device="cuda")
    db.nlines = n
    rc = call_noalloc(torch, db, _lib.FORM_SPLIT)
    assert rc == _lib.SRG_E_ARG
    assert "maximum is 8192" in _lib.last_error()
