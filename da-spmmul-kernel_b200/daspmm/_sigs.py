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


_LL = ctypes.c_longlong
_D = ctypes.c_double


class ServerConfig(ctypes.Structure):
    """daspmm_server_config (include/daspmm.h)."""
    _fields_ = [("budget_bytes", _LL), ("mode", _I), ("val_fmt", _I), ("b_fmt", _I),
                ("chunk", _I), ("max_batch", _I), ("max_inflight", _I), ("window_us", _I),
                ("max_items", _LL), ("scratch_bytes", _LL)]


class Request(ctypes.Structure):
    """daspmm_request (include/daspmm.h)."""
    _fields_ = [("matrix", _I), ("nv", _I), ("B", _VP), ("b_scales", _VP)]


class Result(ctypes.Structure):
    """daspmm_result (include/daspmm.h)."""
    _fields_ = [("status", _I), ("group", _I), ("C", _VP), ("queue_us", _D),
                ("latency_us", _D)]


class ServeStats(ctypes.Structure):
    """daspmm_serve_stats (include/daspmm.h)."""
    _fields_ = [(n, _LL) for n in ("completed", "cancelled", "refused", "groups", "launched",
                                   "items", "queued", "arena_used", "arena_bytes")] + \
               [(n, _I) for n in ("max_group", "inflight_groups", "matrices", "error")]


class MtxHeader(ctypes.Structure):
    """daspmm_mtx_header (include/daspmm.h)."""
    _fields_ = [("nr", _I), ("nc", _I), ("entries", _LL), ("field", _I), ("symmetry", _I),
                ("nnz_max", _LL)]


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
        "daspmm_spmm_host_async": (_I, [ctypes.POINTER(Config), _I, _I, _I, _I, _I, _VP, _VP,
                                        _VP, _VP, _VP, _VP, ctypes.c_float, _VP]),
        "daspmm_launch_count": (ctypes.c_longlong, []),
        "daspmm_spmm_mixed": (_I, [ctypes.POINTER(Config), _I, _I, _I, _I, _I, _VP, _VP, _VP, _I,
                                   _VP, _I, _VP, _VP, ctypes.c_float, _I, _VP, ctypes.c_size_t,
                                   _VP]),
        "daspmm_quantize": (_I, [_I, ctypes.c_size_t, _VP, _VP, _VP, _I, _VP]),
        "daspmm_e4m3_scales": (_I, [_I, _I, _VP, _VP, _VP]),
        "daspmm_device_error": (_I, []),
        "daspmm_wait_probe": (_I, [_I, _I, _VP, _VP]),
        "daspmm_plan_create": (_I, [_VP, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP]),
        "daspmm_plan_spmm": (_I, [_VP, _VP, _VP, ctypes.c_float, _VP]),
        "daspmm_plan_config": (_I, [_VP, _VP]),
        "daspmm_plan_destroy": (_I, [_VP]),
        "daspmm_l2_set_aside": (_I, [ctypes.c_size_t]),
        "daspmm_batch_tune_ex": (_I, [_VP, _I, _VP, _I, _VP, _I, _I, _VP, _VP, _VP]),
        "daspmm_mtx_info": (_I, [ctypes.c_char_p, ctypes.POINTER(MtxHeader)]),
        "daspmm_mtx_read": (_I, [ctypes.c_char_p, _I, _LL, _VP, _VP, _VP, _VP,
                                 ctypes.POINTER(_I)]),
        "daspmm_csr_check": (_I, [_I, _I, _I, _VP, _VP, _I, ctypes.POINTER(_I), _VP]),
        "daspmm_server_create": (_I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]),
        "daspmm_server_add_matrix": (_I, [_VP, _I, _I, _I, _VP, _VP, _VP, ctypes.POINTER(_I)]),
        "daspmm_server_submit": (_I, [_VP, ctypes.POINTER(Request), ctypes.POINTER(_LL)]),
        "daspmm_server_cancel": (_I, [_VP, _LL]),
        "daspmm_server_wait": (_I, [_VP, _LL, _I, ctypes.POINTER(Result)]),
        "daspmm_server_release": (_I, [_VP, _LL]),
        "daspmm_server_replay": (_I, [_VP, ctypes.POINTER(Request), _I, ctypes.POINTER(_D), _I,
                                      ctypes.POINTER(Result)]),
        "daspmm_server_stats": (_I, [_VP, ctypes.POINTER(ServeStats)]),
        "daspmm_server_destroy": (_I, [_VP]),
        "daspmm_kernel_timer_begin": (_I, [_I]),
        "daspmm_kernel_timer_end": (_I, [ctypes.POINTER(ctypes.c_float), _I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
