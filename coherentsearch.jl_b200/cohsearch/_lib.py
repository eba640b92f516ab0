"""ctypes binding of ``libcohsearch_cuda.so`` (declared in ``include/cohsearch.h``).

The library is built in-tree by ``coherentsearch.jl_b200/build.py`` into
``coherentsearch.jl_b200/lib/``.  There is no CPU fallback: if the library is
missing or no CUDA device is present, the calls that need it raise.
"""
import ctypes
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libcohsearch_cuda.so")

CS_OK = 0
CS_ERR_INVALID_ARGUMENT = 1
CS_ERR_NO_SPECTRUM = 2
CS_ERR_CAPACITY = 3
CS_ERR_CUDA = 4
CS_ERR_OUT_OF_MEMORY = 5
CS_ERR_TIMEOUT = 6
CS_ERR_UNSUPPORTED = 7
CS_MAX_DECIM = 16

CS_SYNTH = {"fp32": 0, "bf16": 1, "fp16": 2, "bf16_split": 3, "fp16_split": 4}

STATUS_NAMES = {
    CS_OK: "CS_OK", CS_ERR_INVALID_ARGUMENT: "CS_ERR_INVALID_ARGUMENT",
    CS_ERR_NO_SPECTRUM: "CS_ERR_NO_SPECTRUM", CS_ERR_CAPACITY: "CS_ERR_CAPACITY",
    CS_ERR_CUDA: "CS_ERR_CUDA", CS_ERR_OUT_OF_MEMORY: "CS_ERR_OUT_OF_MEMORY",
    CS_ERR_TIMEOUT: "CS_ERR_TIMEOUT", CS_ERR_UNSUPPORTED: "CS_ERR_UNSUPPORTED",
}


class cs_params(ctypes.Structure):
    _fields_ = [
        ("nharms", ctypes.c_int32),
        ("m", ctypes.c_int32),
        ("numbetween", ctypes.c_int32),
        ("ndecim", ctypes.c_int32),
        ("decimations", ctypes.c_int32 * CS_MAX_DECIM),
        ("hidr", ctypes.c_double),
        ("threshold", ctypes.c_double),
        ("boxcar_fsp", ctypes.c_double),
        ("boxcar_maxfrac", ctypes.c_double),
        ("boxcar_medmargin", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("synth", ctypes.c_int32),
    ]


class cs_candidate(ctypes.Structure):
    _fields_ = [
        ("freq", ctypes.c_double),
        ("metric", ctypes.c_double),
        ("r", ctypes.c_double),
        ("nharm", ctypes.c_int32),
        ("k", ctypes.c_int32),
        ("trial", ctypes.c_int64),
    ]


class cs_spectrum(ctypes.Structure):
    _fields_ = [("amps", ctypes.c_void_p), ("namps", ctypes.c_int64), ("N", ctypes.c_int64),
                ("dt", ctypes.c_double)]


class cs_block_stats(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int64), ("k", ctypes.c_int32), ("Hk", ctypes.c_int32),
                ("nbins", ctypes.c_int32), ("pad", ctypes.c_int32), ("ngoodbins", ctypes.c_double),
                ("flo", ctypes.c_double), ("fhi", ctypes.c_double), ("n", ctypes.c_int64),
                ("min", ctypes.c_double), ("median", ctypes.c_double), ("mean", ctypes.c_double),
                ("std", ctypes.c_double), ("max", ctypes.c_double)]


CAND_DTYPE = np.dtype([("freq", "<f8"), ("metric", "<f8"), ("r", "<f8"), ("nharm", "<i4"),
                       ("k", "<i4"), ("trial", "<i8")])
assert CAND_DTYPE.itemsize == ctypes.sizeof(cs_candidate)


class cs_stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("trials", "blocks", "profiles", "rescued", "candidates", "waves", "launches")] + \
               [(n, ctypes.c_double) for n in
                ("ms_interp", "ms_synth", "ms_sigma", "ms_rescue", "ms_total")] + \
               [(n, ctypes.c_int64) for n in ("h2d_bytes", "d2h_bytes")]


class cs_mlp(ctypes.Structure):
    _fields_ = [("din", ctypes.c_int32), ("dh", ctypes.c_int32), ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p),
                ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p), ("w3", ctypes.c_void_p), ("b3", ctypes.c_void_p)]


class cs_mlp_grads(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("w1", "b1", "w2", "b2", "w3", "b3")]


class cs_adam_param(ctypes.Structure):
    _fields_ = [("master", ctypes.c_void_p), ("bf16", ctypes.c_void_p), ("m", ctypes.c_void_p),
                ("v", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("n", ctypes.c_int64)]


class cs_tune_report(ctypes.Structure):
    _fields_ = [("interp_kernel", ctypes.c_int32), ("sigma_kernel", ctypes.c_int32),
                ("tc_double_buffer", ctypes.c_int32),
                ("tc_div", ctypes.c_int32 * 2), ("nlev", ctypes.c_int32), ("nbins", ctypes.c_int32 * CS_MAX_DECIM),
                ("units", ctypes.c_int32 * CS_MAX_DECIM), ("ms_interp", ctypes.c_double * 2),
                ("ms_sigma", ctypes.c_double * 2),
                ("ms_synth_model", ctypes.c_double), ("ms_synth_tuned", ctypes.c_double),
                ("sample_blocks", ctypes.c_int64)]


_P = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f64 = ctypes.c_double

# name -> (restype, argtypes); every symbol include/cohsearch.h declares.
PROTOTYPES = {
    "cs_create": (_i32, [ctypes.POINTER(_P), ctypes.POINTER(cs_params), _i32]),
    "cs_destroy": (_i32, [_P]),
    "cs_set_stream": (_i32, [_P, _P]),
    "cs_last_error": (ctypes.c_char_p, [_P]),
    "cs_set_spectrum": (_i32, [_P, _P, _i64, _i64, _f64]),
    "cs_set_spectrum_device": (_i32, [_P, _P, _i64, _i64, _f64]),
    "cs_search": (_i32, [_P, _f64, _f64, _i64, _i64, _f64, _i32, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_search_batch": (_i32, [_P, _P, _i32, _i32, _f64, _f64, _i64, _i64, _f64, _P, _P, _i64,
                               ctypes.POINTER(_i64)]),
    "cs_search_range": (_i32, [_P, _f64, _f64, _i64, _i64, _f64, _i32, _i64, _i64, _P, _i64,
                               ctypes.POINTER(_i64)]),
    "cs_search_stats": (_i32, [_P, ctypes.POINTER(cs_stats)]),
    "cs_chunk_metrics": (_i32, [_P, _f64, _i64, _P]),
    "cs_block_metrics": (_i32, [_P, _P, _i64, _i32, _P, _i32, _P]),
    "cs_refold": (_i32, [_P, _P, _P, _i64, _i32, _P, _P, _P]),
    "cs_interp_chunk": (_i32, [_P, _f64, _i64, _i64, _P]),
    "cs_chunk_metrics_static": (_i32, [_P, _P, _i64, _i64, _f64, _i64, _P, _P, _P, _i64]),
    "cs_search_block_values": (_i32, [_P, _P, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_search_trial_metrics": (_i32, [_P, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_set_diagnostics": (_i32, [_P, _i32]),
    "cs_set_memory_limit": (_i32, [_P, _i64]),
    "cs_set_launch_shapes": (_i32, [_P, ctypes.POINTER(cs_tune_report)]),
    "cs_autotune": (_i32, [_P, _f64, _f64, _i64, _i64, _i64, ctypes.POINTER(cs_tune_report)]),
    "cs_set_wait_test": (_i32, [_P, _i64]),
    "cs_search_gate_values": (_i32, [_P, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_version": (ctypes.c_char_p, []),
    "cs_set_metricstats": (_i32, [_P, _i32, _f64, _f64, _i32, _i32]),
    "cs_get_block_stats": (_i32, [_P, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_get_metric_hists": (_i32, [_P, ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(_i32), _P, _P,
                                   _P, _P]),
    "cs_set_metricnorm": (_i32, [_P, _i32, _i32, _P, _P, _P, _P]),
    "cs_set_batch_graph": (_i32, [_P, _i32]),
    "cs_search_blocks": (_i32, [_P, _f64, _f64, _i64, _i64, _f64, _P, _i64, _P, _i64, ctypes.POINTER(_i64)]),
    "cs_block_features": (_i32, [_P, _f64, _f64, _i64, _i64, _P, _i64, ctypes.POINTER(_i64), ctypes.POINTER(_i32)]),
    "cs_mlp_forward": (_i32, [ctypes.POINTER(cs_mlp), _P, _i64, _P, _P, _P, _P]),
    "cs_mlp_backward": (_i32, [ctypes.POINTER(cs_mlp), _P, _P, _P, _P, _P, _i64, ctypes.c_float, _P, _P, _P,
                               ctypes.POINTER(cs_mlp_grads), _P, _P]),
    "cs_adam_step": (_i32, [_P, _i32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _i32, _P]),
    "cs_mlp_to_bf16": (_i32, [_P, _P, _i64, _P]),
}

_lib = None


def load(path=None):
    """Load the library once and bind every prototype; raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libcohsearch_cuda.so not built (expected {p}); "
                           "run coherentsearch.jl_b200/build.py")
    lib = ctypes.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class CohSearchError(RuntimeError):
    """A device or runtime failure reported by the library."""

    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, handle=None, what=""):
    """Map a cs_status to the reference's error behaviour: invalid arguments
    raise ValueError (Julia's ArgumentError), everything else CohSearchError."""
    if status == CS_OK:
        return
    lib = load()
    msg = lib.cs_last_error(handle).decode() if handle else ""
    msg = f"{what}: {msg}" if what else msg
    if status == CS_ERR_INVALID_ARGUMENT:
        raise ValueError(msg or "invalid argument")
    raise CohSearchError(status, msg)
