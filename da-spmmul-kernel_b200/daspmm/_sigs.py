"""ctypes signatures of entry points beyond the core FP32 path.

Kept separate so each added part of the C ABI declares its own signatures in
one place; `apply` skips names the loaded library does not export.
"""
import ctypes

_VP = ctypes.c_void_p
_I = ctypes.c_int


class Instance(ctypes.Structure):
    """daspmm_instance (include/daspmm.h)."""
    _fields_ = [("nr", _I), ("nc", _I), ("nnz", _I), ("nv", _I), ("rowPtr", _VP),
                ("colIdx", _VP), ("values", _VP), ("val_fmt", _I), ("B", _VP), ("b_fmt", _I),
                ("b_scales", _VP), ("C", _VP), ("beta", ctypes.c_float)]


class Fingerprint(ctypes.Structure):
    """daspmm_fingerprint (include/daspmm.h)."""
    _fields_ = [(n, _I) for n in ("layout", "nv", "dtype", "nr", "nnz", "p50", "p90", "p99",
                                  "max_row")]


def apply(lib, Config):
    sig = {
        "daspmm_batch_create": (_I, [ctypes.POINTER(Instance), _I, ctypes.POINTER(Config),
                                     ctypes.POINTER(_VP), _VP]),
        "daspmm_batch_run": (_I, [_VP, _VP]),
        "daspmm_batch_capture": (_I, [_VP, _VP]),
        "daspmm_batch_replay": (_I, [_VP, _VP]),
        "daspmm_batch_info": (_I, [_VP, ctypes.POINTER(ctypes.c_longlong),
                                   ctypes.POINTER(ctypes.c_longlong)]),
        "daspmm_batch_destroy": (_I, [_VP]),
        "daspmm_batch_tune": (_I, [ctypes.POINTER(Instance), _I, _VP, _I, _I,
                                   ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float), _VP]),
        "daspmm_autotune": (_I, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP, _I,
                                 ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_float), _VP]),
        "daspmm_fingerprint_of": (_I, [_I, _I, _I, _I, _I, _VP, _VP,
                                       ctypes.POINTER(Fingerprint)]),
        "daspmm_tune_save": (_I, [ctypes.c_char_p]),
        "daspmm_tune_load": (_I, [ctypes.c_char_p]),
        "daspmm_tune_clear": (None, []),
        "daspmm_spmm_host": (_I, [ctypes.POINTER(Config), _I, _I, _I, _I, _I, _VP, _VP, _VP,
                                  _VP, _VP, _VP, ctypes.c_float, _VP]),
        "daspmm_launch_count": (ctypes.c_longlong, []),
        "daspmm_spmm_mixed": (_I, [ctypes.POINTER(Config), _I, _I, _I, _I, _I, _VP, _VP, _VP, _I,
                                   _VP, _I, _VP, _VP, ctypes.c_float, _I, _VP, ctypes.c_size_t,
                                   _VP]),
        "daspmm_quantize": (_I, [_I, ctypes.c_size_t, _VP, _VP, _VP, _I, _VP]),
        "daspmm_e4m3_scales": (_I, [_I, _I, _VP, _VP, _VP]),
        "daspmm_device_error": (_I, []),
        "daspmm_kernel_timer_begin": (_I, [_I]),
        "daspmm_kernel_timer_end": (_I, [ctypes.POINTER(ctypes.c_float), _I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
