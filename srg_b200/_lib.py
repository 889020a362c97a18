"""ctypes view of libsrg_bp.so (include/srg_bp.h).

The library is the product: every backprojection in this package runs
through it.  Loading fails loudly when it is missing; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsrg_bp.so")

SRG_OK = 0
SRG_E_ARG = -1
SRG_E_CUDA = -2
SRG_E_IO = -3
SRG_E_TIMEOUT = -4
SRG_E_NOMEM = -5
SRG_E_UNSUPPORTED = -6

FORM_FP64 = 0
FORM_SPLIT = 1
TILE_SHEAR_AUTO = 1000   # srg_bp_options.tile_shear: chosen from the geometry
MAX_TILE_SHEAR = 8

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class Options(C.Structure):
    _fields_ = [("form", C.c_int), ("tile_cfg", C.c_int), ("device", C.c_int),
                ("centres_on_host", C.c_int), ("verbose", C.c_int), ("spin_limit", C.c_int),
                ("full_lines", C.c_int), ("scratch_limit", C.c_longlong), ("overlap", C.c_int),
                ("tile_shear", C.c_int)]


class BurstDesc(C.Structure):
    _fields_ = [
        ("burst", C.c_void_p), ("satloc", C.c_void_p), ("dem", C.c_void_p), ("out", C.c_void_p),
        ("coef", C.c_void_p),
        ("ldb", C.c_int64), ("dem_ld", C.c_int64), ("out_ld", C.c_int64),
        ("P", C.c_int), ("S", C.c_int), ("demwidth", C.c_int),
        ("firstline", C.c_int), ("nlines", C.c_int), ("firstpix", C.c_int), ("lastpix", C.c_int),
        ("out_pix0", C.c_int), ("aperture", C.c_int),
        ("firstlat", C.c_double), ("deltalat", C.c_double), ("firstlon", C.c_double),
        ("deltalon", C.c_double),
        ("rngstart", C.c_double), ("rngend", C.c_double), ("dmrg", C.c_double), ("wvl", C.c_double),
        ("timeorbit", _dp), ("xx", _dp), ("vv", _dp),
        ("numstatevec", C.c_int),
        ("tmid", C.c_double), ("xyz_mid", C.c_double * 3), ("vel_mid", C.c_double * 3),
        ("angc0", C.c_double), ("angc1", C.c_double), ("prf", C.c_double),
        ("bin0", C.c_int), ("nbins", C.c_int),
    ]


class BurstParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "starttime", "prf", "samplefreq", "pri", "range0", "wvl", "angc0", "angc1", "tstart",
        "tend", "tmid", "dtaz", "rngstart", "rngend", "dmrg")] + [("aperture", C.c_int),
                                                                 ("pad", C.c_int)]


INTERP_LINEAR = 0
INTERP_OVERSAMPLED2 = 1


class TuneRequest(C.Structure):
    _fields_ = [("iters", C.c_int), ("use_cache", C.c_int), ("interp_budget", C.c_double)]


class TuneResult(C.Structure):
    _fields_ = [("tile_cfg", C.c_int), ("interp", C.c_int), ("from_cache", C.c_int),
                ("tile_shear", C.c_int), ("ms", C.c_double), ("err_linear", C.c_double),
                ("err_oversampled", C.c_double)]


class SrgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"srg error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

_SIGS = {
    "srg_bp_default_options": (None, [C.POINTER(Options)]),
    "srg_last_error": (C.c_char_p, []),
    "srg_set_default_options": (None, [C.POINTER(Options)]),
    "srg_bp_bursts_device": (C.c_int, [C.POINTER(BurstDesc), C.c_int, C.POINTER(Options), C.c_void_p]),
    "srg_count_terms_device": (C.c_int, [C.POINTER(BurstDesc), C.c_int, C.POINTER(C.c_int64), C.c_void_p]),
    "srg_merge_device": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p]),
    "srg_line_centres_device": (C.c_int, [C.POINTER(BurstDesc), C.c_void_p, C.c_void_p]),
    "srg_pulse_orbit_device": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "srg_sync_check": (C.c_int, [C.c_void_p]),
    "srg_bp_burst_device_gated": (C.c_int, [C.POINTER(BurstDesc), C.c_void_p, C.c_int, C.c_int,
                                            C.POINTER(Options), C.c_void_p]),
    "srg_test_set_dropin_sequence": (C.c_int, [C.c_int, C.c_int]),
    "srg_dropin_flush": (C.c_int, [C.c_int]),
    "srg_dropin_last_bytes": (C.c_int, [C.c_int, C.POINTER(C.c_longlong),
                                        C.POINTER(C.c_longlong)]),
    "srg_burst_params": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_int, _dp,
                                   C.POINTER(BurstParams)]),
    "srg_measure_fma_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "srg_bp_burst_device_noalloc": (C.c_int, [C.POINTER(BurstDesc), C.POINTER(Options), C.c_void_p]),
    "srg_scene_create": (C.c_int, [C.POINTER(BurstDesc), C.c_int, C.c_void_p, C.c_int64, C.c_int,
                                   C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "srg_scene_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "srg_scene_sync": (C.c_int, [C.c_void_p, C.c_void_p]),
    "srg_scene_run_stages": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "srg_scene_terms": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "srg_scene_tune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "srg_scene_autotune": (C.c_int, [C.c_void_p, C.POINTER(TuneRequest), C.POINTER(TuneResult)]),
    "srg_scene_set_interp": (C.c_int, [C.c_void_p, C.c_int]),
    "srg_scene_interp": (C.c_int, [C.c_void_p]),
    "srg_interp_error": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    "srg_scene_set_shape": (C.c_int, [C.c_void_p, C.c_int]),
    "srg_scene_set_form": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "srg_scene_shape": (C.c_int, [C.c_void_p]),
    "srg_scene_tile_shear": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "srg_scene_destroy": (None, [C.c_void_p]),
    "srg_tile_config_count": (C.c_int, []),
    "srg_tile_shear": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "srg_tile_config": (C.c_int, [C.c_int, _ip, _ip, _ip, _ip, _ip]),
    "srg_tile_config_name": (C.c_char_p, [C.c_int]),
    "srg_forward_project_device": (C.c_int, [C.POINTER(BurstDesc), C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_double, C.c_void_p, C.c_void_p]),
    "srg_crossmul_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "srg_crossmul_stack_device": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_longlong, C.c_int,
                                            C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                            C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p]),
    "srg_range_replica": (C.c_int, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_int,
                                    _ip]),
    "srg_range_compress_device": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_float,
                                            C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_longlong,
                                            _ip, C.c_void_p]),
    "srg_oversample_taps": (None, [C.c_void_p]),
    "srg_oversample_range_device": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_void_p,
                                              C.c_longlong, C.c_void_p]),
    "srg_azimuth_compress": (C.c_int, [
        _fp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
        C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp, C.c_int,
        C.c_double, C.c_double, C.c_double, _dp, _dp, C.c_double, C.c_double, C.c_int,
        C.c_double, C.c_double, C.c_double, C.POINTER(Options)]),
}

EXPORTS = tuple(_SIGS) + ("azimuth_compress_",)


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"{LIB_PATH} is missing: build it with `python -m srg_b200.build`")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            L.azimuth_compress_.restype = None
            _lib = L
        return _lib


def last_error() -> str:
    return lib().srg_last_error().decode()


def check(rc: int) -> None:
    if rc != SRG_OK:
        raise SrgError(rc, last_error())


def default_options(form: int = FORM_SPLIT, tile_cfg: int = -1, device: int = -1) -> Options:
    o = Options()
    lib().srg_bp_default_options(C.byref(o))
    o.form = form
    o.tile_cfg = tile_cfg
    o.device = device
    return o


def measure_fma_peak(fp64: bool) -> float:
    v = C.c_double()
    check(lib().srg_measure_fma_peak(1 if fp64 else 0, C.byref(v)))
    return float(v.value)


def tile_config_name(idx: int) -> str:
    return lib().srg_tile_config_name(idx).decode()


def tile_configs():
    """[(index, form, tile_x, tile_y, threads, chunk, window)]."""
    L = lib()
    out = []
    for i in range(L.srg_tile_config_count()):
        v = [C.c_int() for _ in range(5)]
        form = L.srg_tile_config(i, *[C.byref(x) for x in v])
        out.append((i, form) + tuple(x.value for x in v))
    return out
