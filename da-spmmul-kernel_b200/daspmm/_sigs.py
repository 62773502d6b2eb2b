"""ctypes signatures of entry points beyond the core FP32 path.

Kept separate so each added part of the C ABI declares its own signatures in
one place; `apply` skips names the loaded library does not export.
"""
import ctypes

_VP = ctypes.c_void_p
_I = ctypes.c_int


def apply(lib, Config):
    sig = {
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
