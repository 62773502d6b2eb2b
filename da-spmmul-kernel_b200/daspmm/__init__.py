"""Python bindings of libdaspmm.so (the C ABI in include/daspmm.h).

ctypes over the shared library; torch tensors supply device memory and
streams only.  Loading fails loudly when the library has not been built --
there is no CPU fallback for any computation here.

Mirrors the reference's host interface (ASPLOS-2022/DA-SpMMul-kernel):
``SPMV_SPMM_ALG`` (spmvspmm.h:5-10), ``DenseLayout`` (helper.h:261-264),
``SpmvSpmmProblem`` (spmvspmm.h:13-50, 202-273) and ``cudaSpmm``
(spmvspmm.h:53-199).
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libdaspmm.so")


class DaspmmError(RuntimeError):
    """A libdaspmm call returned a non-zero status."""

    def __init__(self, status: int, what: str = ""):
        self.status = int(status)
        msg = _lib().daspmm_status_string(int(status)).decode()
        if self.status == 3:
            msg += f" (cudaError {_lib().daspmm_last_cuda_error()})"
        super().__init__(f"{what}: {msg}" if what else msg)


class Alg(enum.IntEnum):
    """SPMV_SPMM_ALG (spmvspmm.h:5-10) plus this library's extensions."""

    CSR_SCALAR = 0
    CSR_VECTOR = 1
    COO_SCALAR = 2
    COO_VECTOR = 3
    CSR_BALANCED = 4
    AUTO = 5


class Layout(enum.IntEnum):
    """DenseLayout (helper.h:261-264)."""

    ROW_MAJOR = 0
    COL_MAJOR = 1


class Fmt(enum.IntEnum):
    F32 = 0
    BF16 = 1
    F16 = 2
    E4M3 = 3


class Config(ctypes.Structure):
    """daspmm_config: one point of the design space (0 = library default)."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("alg", "vec", "lanes_col", "lanes_nnz", "cf", "chunk", "snap", "block", "pipe",
                 "l2_window")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}

    def __repr__(self):
        return "Config(" + ", ".join(f"{k}={v}" for k, v in self.as_dict().items()) + ")"


_LIB = None
_VP = ctypes.c_void_p
_I = ctypes.c_int


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C {os.path.dirname(_HERE)}` "
                "(or __graft_entry__.build()); there is no fallback implementation")
        lib = ctypes.CDLL(LIB_PATH)
        sig = {
            "daspmm_spmm": (_I, [_I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP,
                                 ctypes.c_float, _VP]),
            "daspmm_spmm_ex": (_I, [ctypes.POINTER(Config), _I, _I, _I, _I, _I, _VP, _VP, _VP,
                                    _VP, _VP, _VP, ctypes.c_float, _VP, ctypes.c_size_t, _VP]),
            "daspmm_workspace_bytes": (ctypes.c_size_t,
                                       [ctypes.POINTER(Config), _I, _I, _I, _I, _I]),
            "daspmm_default_config": (_I, [_I, _I, _I, _I, _I, _I, ctypes.POINTER(Config)]),
            "daspmm_compat_spmm": (_I, [_I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
            "daspmm_num_chunks": (_I, [_I, _I]),
            "daspmm_partition": (_I, [_I, _I, _VP, _I, _I, _VP, _VP]),
            "daspmm_ownership": (_I, [_I, _I, _I, _VP, _VP, _I, _I, _VP, _VP]),
            "daspmm_coo_to_csr": (_I, [_I, _I, _VP, _VP, _VP]),
            "daspmm_status_string": (ctypes.c_char_p, [_I]),
            "daspmm_last_cuda_error": (_I, []),
            "daspmm_abi_version": (_I, []),
            "daspmm_gen_uniform": (_I, [_I, _I, _I, ctypes.c_uint64, _VP, _VP, _VP]),
            "daspmm_gen_powerlaw": (_I, [_I, _I, ctypes.c_double, ctypes.c_double, _I, _I,
                                         ctypes.c_double, ctypes.c_uint64, _VP, _VP, _VP,
                                         ctypes.POINTER(ctypes.c_longlong)]),
            "daspmm_gen_random": (_I, [_I, _I, ctypes.c_double, ctypes.c_uint64, _VP, _VP, _VP,
                                       ctypes.POINTER(ctypes.c_longlong)]),
            "daspmm_gen_dense": (None, [ctypes.c_size_t, ctypes.c_uint64, ctypes.c_float,
                                        ctypes.c_float, _VP]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _extend_signatures(lib)
        _LIB = lib
    return _LIB


def _extend_signatures(lib):
    """Signatures of entry points added by later modules of the library."""
    from . import _sigs
    _sigs.apply(lib, Config)


def lib():
    """The loaded libdaspmm.so (ctypes.CDLL)."""
    return _lib()


def check(status: int, what: str = "") -> None:
    if status != 0:
        raise DaspmmError(status, what)


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


# ---------------------------------------------------------------- matrices
@dataclass
class Csr:
    """Host CSR matrix (int32 indices, float32 values), sorted by (row, col)."""

    nr: int
    nc: int
    rowPtr: np.ndarray
    colIdx: np.ndarray
    values: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowPtr[-1]) if self.nr > 0 else 0

    @property
    def rowIdx(self) -> np.ndarray:
        """COO row indices (the reference driver passes both, spmvspmm_benchmark.cu:370)."""
        return np.repeat(np.arange(self.nr, dtype=np.int32), np.diff(self.rowPtr)).astype(np.int32)

    def cols_touched(self) -> int:
        return int(np.unique(self.colIdx).size) if self.nnz else 0


def gen_uniform(nr: int, nc: int, per_row: int, seed: int = 0) -> Csr:
    """Exactly per_row distinct uniform columns per row, values U(-1,1)."""
    L = _lib()
    rp = np.zeros(nr + 1, np.int32)
    ci = np.zeros(max(1, nr * per_row), np.int32)
    va = np.zeros(max(1, nr * per_row), np.float32)
    check(L.daspmm_gen_uniform(nr, nc, per_row, seed, _np_ptr(rp), _np_ptr(ci), _np_ptr(va)),
          "gen_uniform")
    n = nr * per_row
    return Csr(nr, nc, rp, ci[:n].copy(), va[:n].copy())


def gen_powerlaw(n: int, alpha: float = 2.1, shift: float = 0.16, dmin: int = 1,
                 dmax: int = 4096, seed: int = 0, mean_scale: float = 1.0,
                 nc: int | None = None) -> Csr:
    """Power-law out-degrees, preferential-attachment columns, values U(-1,1)."""
    L = _lib()
    nc = n if nc is None else nc
    rp = np.zeros(n + 1, np.int32)
    nnz = ctypes.c_longlong(0)
    check(L.daspmm_gen_powerlaw(n, nc, alpha, shift, dmin, dmax, mean_scale, seed,
                                _np_ptr(rp), None, None, ctypes.byref(nnz)), "gen_powerlaw")
    ci = np.zeros(max(1, nnz.value), np.int32)
    va = np.zeros(max(1, nnz.value), np.float32)
    check(L.daspmm_gen_powerlaw(n, nc, alpha, shift, dmin, dmax, mean_scale, seed,
                                _np_ptr(rp), _np_ptr(ci), _np_ptr(va), ctypes.byref(nnz)),
          "gen_powerlaw")
    return Csr(n, nc, rp, ci[:nnz.value].copy(), va[:nnz.value].copy())


def gen_random(nr: int, nc: int, avg_deg: float, seed: int = 0) -> Csr:
    """Poisson(avg_deg) distinct uniform columns per row, values U(-1,1)."""
    L = _lib()
    rp = np.zeros(nr + 1, np.int32)
    nnz = ctypes.c_longlong(0)
    check(L.daspmm_gen_random(nr, nc, avg_deg, seed, _np_ptr(rp), None, None,
                              ctypes.byref(nnz)), "gen_random")
    ci = np.zeros(max(1, nnz.value), np.int32)
    va = np.zeros(max(1, nnz.value), np.float32)
    check(L.daspmm_gen_random(nr, nc, avg_deg, seed, _np_ptr(rp), _np_ptr(ci), _np_ptr(va),
                              ctypes.byref(nnz)), "gen_random")
    return Csr(nr, nc, rp, ci[:nnz.value].copy(), va[:nnz.value].copy())


def gen_dense(n: int, seed: int = 1, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(max(1, n), np.float32)
    _lib().daspmm_gen_dense(n, seed, lo, hi, _np_ptr(out))
    return out[:n]


def default_config(alg: int, layout: int, nr: int, nc: int, nnz: int, nv: int) -> Config:
    c = Config()
    check(_lib().daspmm_default_config(int(alg), int(layout), nr, nc, nnz, nv, ctypes.byref(c)),
          "default_config")
    return c


def num_chunks(nnz: int, chunk: int) -> int:
    return _lib().daspmm_num_chunks(nnz, chunk)


def workspace_bytes(cfg: Config, layout: int, nr: int, nc: int, nnz: int, nv: int) -> int:
    return _lib().daspmm_workspace_bytes(ctypes.byref(cfg), int(layout), nr, nc, nnz, nv)


# ---------------------------------------------------------------- device side
def _dptr(t):
    """Device address of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(getattr(stream, "cuda_stream", stream))


class DeviceCsr:
    """A CSR/COO matrix resident in device memory (torch tensors)."""

    def __init__(self, A: Csr, device="cuda"):
        import torch
        self.nr, self.nc, self.nnz = A.nr, A.nc, A.nnz
        self.rowPtr = torch.from_numpy(A.rowPtr).to(device)
        self.rowIdx = torch.from_numpy(A.rowIdx).to(device)
        self.colIdx = torch.from_numpy(A.colIdx).to(device)
        self.values = torch.from_numpy(A.values).to(device)


def spmm(alg: int, layout: int, A: DeviceCsr, B, C, beta: float = 0.0, nv: int | None = None,
         stream=None, cfg: Config | None = None, workspace=None) -> None:
    """C = A*B + beta*C on the device (libdaspmm.daspmm_spmm / daspmm_spmm_ex)."""
    L = _lib()
    if nv is None:
        nv = B.shape[1] if (layout == Layout.ROW_MAJOR and B.dim() == 2) else (
            B.shape[0] if B.dim() == 2 else 1)
    if cfg is None:
        st = L.daspmm_spmm(int(alg), int(layout), A.nr, A.nc, A.nnz, nv, _dptr(A.rowPtr),
                           _dptr(A.rowIdx), _dptr(A.colIdx), _dptr(A.values), _dptr(B), _dptr(C),
                           float(beta), _stream_ptr(stream))
    else:
        ws = _dptr(workspace)
        wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
        st = L.daspmm_spmm_ex(ctypes.byref(cfg), int(layout), A.nr, A.nc, A.nnz, nv,
                              _dptr(A.rowPtr), _dptr(A.rowIdx), _dptr(A.colIdx), _dptr(A.values),
                              _dptr(B), _dptr(C), float(beta), ws, wsb, _stream_ptr(stream))
    check(st, "daspmm_spmm")


def compat_spmm(alg: int, layout: int, A: DeviceCsr, B, C, nv: int) -> int:
    """cudaSpmm<256,32> semantics (CSR overwrite, COO accumulate); returns cudaError_t."""
    return _lib().daspmm_compat_spmm(int(alg), int(layout), A.nr, A.nc, A.nnz, nv,
                                     _dptr(A.rowPtr), _dptr(A.rowIdx), _dptr(A.colIdx),
                                     _dptr(A.values), _dptr(B), _dptr(C))


def partition(A: DeviceCsr, chunk: int, snap: int, stream=None):
    import torch
    n = num_chunks(A.nnz, chunk)
    meta = torch.empty(2 * (n + 1), dtype=torch.int32, device=A.rowPtr.device)
    check(_lib().daspmm_partition(A.nr, A.nnz, _dptr(A.rowPtr), chunk, snap, _dptr(meta),
                                  _stream_ptr(stream)), "partition")
    return meta


def ownership(alg: int, A: DeviceCsr, chunk: int, snap: int = 1, stream=None):
    import torch
    own = torch.empty(2 * max(1, A.nr), dtype=torch.int32, device=A.rowPtr.device)
    check(_lib().daspmm_ownership(int(alg), A.nr, A.nnz, _dptr(A.rowPtr), _dptr(A.rowIdx),
                                  chunk, snap, _dptr(own), _stream_ptr(stream)), "ownership")
    return own[: 2 * A.nr]


def coo_to_csr(nr: int, rowIdx, stream=None):
    import torch
    rp = torch.empty(nr + 1, dtype=torch.int32, device=rowIdx.device)
    check(_lib().daspmm_coo_to_csr(nr, rowIdx.numel(), _dptr(rowIdx), _dptr(rp),
                                   _stream_ptr(stream)), "coo_to_csr")
    return rp


# ---------------------------------------------------------------- mixed precision
_TORCH_STORE = {Fmt.BF16: "bfloat16", Fmt.F16: "float16", Fmt.E4M3: "uint8"}


def quantize(x, fmt: int, col_scales=None, ncols: int = 0, stream=None):
    """Device round-to-nearest-even of an FP32 tensor to BF16 / FP16 / E4M3
    (E4M3 returned as uint8 codes), optionally dividing by per-column scales."""
    import torch
    fmt = Fmt(fmt)
    q = torch.empty(x.numel(), dtype=getattr(torch, _TORCH_STORE[fmt]), device=x.device)
    check(_lib().daspmm_quantize(int(fmt), x.numel(), _dptr(x), _dptr(q), _dptr(col_scales),
                                 ncols, _stream_ptr(stream)), "quantize")
    return q


def e4m3_scales(B, nrows: int, ncols: int, stream=None):
    """Per-column FP32 scales max|B[:,k]|/448 of a row-major FP32 matrix."""
    import torch
    s = torch.empty(ncols, dtype=torch.float32, device=B.device)
    check(_lib().daspmm_e4m3_scales(nrows, ncols, _dptr(B), _dptr(s), _stream_ptr(stream)),
          "e4m3_scales")
    return s


def spmm_mixed(A: DeviceCsr, values, val_fmt: int, B, b_fmt: int, C, nv: int,
               b_scales=None, beta: float = 0.0, kahan_min: int = 0, cfg: Config | None = None,
               stream=None) -> None:
    """C (FP32) = A*B + beta*C with values / B in reduced-precision storage."""
    check(_lib().daspmm_spmm_mixed(ctypes.byref(cfg) if cfg is not None else None, 0, A.nr,
                                   A.nc, A.nnz, nv, _dptr(A.rowPtr), _dptr(A.colIdx),
                                   _dptr(values), int(val_fmt), _dptr(B), int(b_fmt),
                                   _dptr(b_scales), _dptr(C), float(beta), int(kahan_min), None,
                                   0, _stream_ptr(stream)), "spmm_mixed")


# ---------------------------------------------------------------- autotuner
def autotune(layout: int, A: DeviceCsr, B, C, nv: int, reps: int = 5, use_coo: bool = True,
             stream=None):
    """Times the design-space candidates on this problem and caches the best
    for DASPMM_ALG_AUTO; returns (Config, microseconds per call)."""
    cfg = Config()
    us = ctypes.c_float()
    check(_lib().daspmm_autotune(int(layout), A.nr, A.nc, A.nnz, nv, _dptr(A.rowPtr),
                                 _dptr(A.rowIdx) if use_coo else None, _dptr(A.colIdx),
                                 _dptr(A.values), _dptr(B), _dptr(C), reps, ctypes.byref(cfg),
                                 ctypes.byref(us), _stream_ptr(stream)), "autotune")
    return cfg, us.value


def fingerprint(layout: int, A: DeviceCsr, nv: int, dtype: int = 0, stream=None) -> dict:
    from ._sigs import Fingerprint
    fp = Fingerprint()
    check(_lib().daspmm_fingerprint_of(int(layout), A.nr, A.nnz, nv, dtype, _dptr(A.rowPtr),
                                       _stream_ptr(stream), ctypes.byref(fp)), "fingerprint")
    return {n: getattr(fp, n) for n, _ in fp._fields_}


# ---------------------------------------------------------------- batches
class Plan:
    """daspmm_plan_*: one matrix (a DeviceCsr that must outlive the plan), row-
    major, nv columns; the balanced split's boundaries computed once, each
    product one launch of the window kernel (bit-identical to spmm with the
    same configuration)."""

    def __init__(self, A: DeviceCsr, nv: int, cfg: Config | None = None, stream=None):
        self.A, self.nv = A, int(nv)
        self._h = ctypes.c_void_p()
        check(_lib().daspmm_plan_create(ctypes.byref(cfg) if cfg is not None else None, A.nr,
                                        A.nc, A.nnz, self.nv, _dptr(A.rowPtr), _dptr(A.colIdx),
                                        _dptr(A.values), _stream_ptr(stream),
                                        ctypes.byref(self._h)), "plan_create")

    def spmm(self, B, C, beta: float = 0.0, stream=None) -> None:
        check(_lib().daspmm_plan_spmm(self._h, _dptr(B), _dptr(C), float(beta),
                                      _stream_ptr(stream)), "plan_spmm")

    def config(self) -> Config:
        c = Config()
        check(_lib().daspmm_plan_config(self._h, ctypes.byref(c)), "plan_config")
        return c

    def close(self):
        if self._h:
            _lib().daspmm_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many SpMMs in one persistent launch (daspmm_batch_*).

    `instances` is a list of dicts with keys A (DeviceCsr), values (device
    tensor, F32 or BF16), B, C (device tensors), nv, optional val_fmt, b_fmt,
    b_scales, beta.  The tensors must outlive the batch."""

    def __init__(self, instances, chunk: int = 0, stream=None, lanes_col: int = 0):
        from ._sigs import Instance
        self._keep = instances
        arr = (Instance * max(1, len(instances)))()
        for i, d in enumerate(instances):
            A = d["A"]
            arr[i] = Instance(A.nr, A.nc, A.nnz, d["nv"], _dptr(A.rowPtr) or 0,
                              _dptr(A.colIdx) or 0, _dptr(d.get("values", A.values)) or 0,
                              int(d.get("val_fmt", Fmt.F32)), _dptr(d["B"]) or 0,
                              int(d.get("b_fmt", Fmt.F32)), _dptr(d.get("b_scales")) or 0,
                              _dptr(d["C"]) or 0, float(d.get("beta", 0.0)))
        self._h = ctypes.c_void_p()
        cfg = Config(chunk=chunk, lanes_col=lanes_col)
        check(_lib().daspmm_batch_create(arr, len(instances), ctypes.byref(cfg),
                                         ctypes.byref(self._h), _stream_ptr(stream)),
              "batch_create")

    def run(self, stream=None):
        check(_lib().daspmm_batch_run(self._h, _stream_ptr(stream)), "batch_run")

    def capture(self, stream):
        check(_lib().daspmm_batch_capture(self._h, _stream_ptr(stream)), "batch_capture")

    def replay(self, stream):
        check(_lib().daspmm_batch_replay(self._h, _stream_ptr(stream)), "batch_replay")

    @staticmethod
    def tune(instances, chunks=None, reps: int = 5, stream=None):
        """Fastest row-tile size for this set of instances: (chunk, us)."""
        from ._sigs import Instance
        arr = (Instance * max(1, len(instances)))()
        for i, d in enumerate(instances):
            A = d["A"]
            arr[i] = Instance(A.nr, A.nc, A.nnz, d["nv"], _dptr(A.rowPtr) or 0,
                              _dptr(A.colIdx) or 0, _dptr(d.get("values", A.values)) or 0,
                              int(d.get("val_fmt", Fmt.F32)), _dptr(d["B"]) or 0,
                              int(d.get("b_fmt", Fmt.F32)), _dptr(d.get("b_scales")) or 0,
                              _dptr(d["C"]) or 0, float(d.get("beta", 0.0)))
        ch = (ctypes.c_int * len(chunks))(*chunks) if chunks else None
        best, us = ctypes.c_int(), ctypes.c_float()
        check(_lib().daspmm_batch_tune(arr, len(instances), ch, len(chunks) if chunks else 0,
                                       reps, ctypes.byref(best), ctypes.byref(us),
                                       _stream_ptr(stream)), "batch_tune")
        return best.value, us.value

    @staticmethod
    def tune_ex(instances, chunks=None, widths=None, reps: int = 5, stream=None):
        """Fastest (row-tile size, column-tile width) for these instances:
        (Config with chunk and lanes_col, us)."""
        from ._sigs import Instance
        arr = (Instance * max(1, len(instances)))()
        for i, d in enumerate(instances):
            A = d["A"]
            arr[i] = Instance(A.nr, A.nc, A.nnz, d["nv"], _dptr(A.rowPtr) or 0,
                              _dptr(A.colIdx) or 0, _dptr(d.get("values", A.values)) or 0,
                              int(d.get("val_fmt", Fmt.F32)), _dptr(d["B"]) or 0,
                              int(d.get("b_fmt", Fmt.F32)), _dptr(d.get("b_scales")) or 0,
                              _dptr(d["C"]) or 0, float(d.get("beta", 0.0)))
        ch = (ctypes.c_int * len(chunks))(*chunks) if chunks else None
        wd = (ctypes.c_int * len(widths))(*widths) if widths else None
        best, us = Config(), ctypes.c_float()
        check(_lib().daspmm_batch_tune_ex(arr, len(instances), ch, len(chunks) if chunks else 0,
                                          wd, len(widths) if widths else 0, reps,
                                          ctypes.byref(best), ctypes.byref(us),
                                          _stream_ptr(stream)), "batch_tune_ex")
        return best, us.value

    def info(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(_lib().daspmm_batch_info(self._h, ctypes.byref(a), ctypes.byref(b)), "batch_info")
        return a.value, b.value

    def close(self):
        if self._h:
            _lib().daspmm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- Matrix Market
def mtx_info(path: str) -> dict:
    from ._sigs import MtxHeader
    h = MtxHeader()
    check(_lib().daspmm_mtx_info(os.fsencode(path), ctypes.byref(h)), f"mtx_info {path}")
    return {n: getattr(h, n) for n, _ in h._fields_}


def read_mtx(path: str, keep_diagonal: bool = False) -> Csr:
    """A Matrix Market coordinate file as a sorted CSR (daspmm_mtx_read)."""
    h = mtx_info(path)
    cap = int(h["nnz_max"])
    rp = np.zeros(h["nr"] + 1, np.int32)
    ci = np.zeros(max(1, cap), np.int32)
    va = np.zeros(max(1, cap), np.float32)
    n = ctypes.c_int()
    check(_lib().daspmm_mtx_read(os.fsencode(path), 1 if keep_diagonal else 0, cap,
                                 rp.ctypes.data, None, ci.ctypes.data, va.ctypes.data,
                                 ctypes.byref(n)), f"mtx_read {path}")
    return Csr(h["nr"], h["nc"], rp, ci[: n.value].copy(), va[: n.value].copy())


# ---------------------------------------------------------------- validation
def csr_check(A: DeviceCsr, sorted_cols: bool = False, stream=None) -> int:
    """-1 when A passes daspmm_csr_check, else the first offending row."""
    bad = ctypes.c_int(-1)
    st = _lib().daspmm_csr_check(A.nr, A.nc, A.nnz, _dptr(A.rowPtr), _dptr(A.colIdx),
                                 int(bool(sorted_cols)), ctypes.byref(bad), _stream_ptr(stream))
    if st == 9:
        return bad.value
    check(st, "csr_check")
    return -1


# ---------------------------------------------------------------- serving
class ServeMode(enum.IntEnum):
    BATCHED = 0
    PLAIN = 1


class _DeviceView:
    """A raw device float32 buffer as a torch tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None}


class Server:
    """daspmm_server_*: a pool of resident matrices, an output arena and a
    dispatcher thread.  Matrices (DeviceCsr + values tensor) and every
    request's B must outlive the server's use of them."""

    def __init__(self, budget_bytes: int = 1 << 30, mode: int = ServeMode.BATCHED,
                 val_fmt: int = Fmt.F32, b_fmt: int = Fmt.F32, chunk: int = 0,
                 max_batch: int = 0, max_inflight: int = 0, window_us: int = 0,
                 max_items: int = 0, scratch_bytes: int = 0):
        from ._sigs import ServerConfig
        cfg = ServerConfig(int(budget_bytes), int(mode), int(val_fmt), int(b_fmt), chunk,
                           max_batch, max_inflight, window_us, max_items, scratch_bytes)
        self._h = ctypes.c_void_p()
        check(_lib().daspmm_server_create(ctypes.byref(cfg), ctypes.byref(self._h)),
              "server_create")
        self._keep = []
        self.shapes = []

    def add_matrix(self, A: DeviceCsr, values=None) -> int:
        mid = ctypes.c_int(-1)
        v = A.values if values is None else values
        check(_lib().daspmm_server_add_matrix(self._h, A.nr, A.nc, A.nnz, _dptr(A.rowPtr),
                                              _dptr(A.colIdx), _dptr(v), ctypes.byref(mid)),
              "server_add_matrix")
        self._keep.append((A, v))
        self.shapes.append((A.nr, A.nc, A.nnz))
        return mid.value

    @staticmethod
    def _req(matrix: int, nv: int, B, b_scales=None):
        from ._sigs import Request
        return Request(int(matrix), int(nv), _dptr(B) or 0, _dptr(b_scales) or 0)

    def submit(self, matrix: int, nv: int, B, b_scales=None) -> int:
        t = ctypes.c_longlong()
        r = self._req(matrix, nv, B, b_scales)
        check(_lib().daspmm_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)),
              "server_submit")
        return t.value

    def cancel(self, ticket: int) -> int:
        return _lib().daspmm_server_cancel(self._h, int(ticket))

    def wait(self, ticket: int, timeout_ms: int = -1):
        from ._sigs import Result
        r = Result()
        st = _lib().daspmm_server_wait(self._h, int(ticket), int(timeout_ms), ctypes.byref(r))
        return st, r

    def result_tensor(self, res, nrows: int, nv: int):
        """The result's C (device, FP32) as a torch tensor view; valid until release."""
        import torch
        if not res.C:
            return None
        return torch.as_tensor(_DeviceView(res.C, nrows * nv), device="cuda")

    def release(self, ticket: int) -> None:
        check(_lib().daspmm_server_release(self._h, int(ticket)), "server_release")

    def replay(self, requests, arrivals, release: bool = True):
        """requests: list of (matrix, nv, B[, b_scales]); arrivals: seconds."""
        from ._sigs import Request, Result
        n = len(requests)
        arr = (Request * max(1, n))()
        for i, q in enumerate(requests):
            arr[i] = self._req(*q)
        ts = (ctypes.c_double * max(1, n))(*[float(a) for a in arrivals])
        res = (Result * max(1, n))()
        st = _lib().daspmm_server_replay(self._h, arr, n, ts, int(bool(release)), res)
        check(st, "server_replay")
        return [res[i] for i in range(n)]

    def stats(self) -> dict:
        from ._sigs import ServeStats
        o = ServeStats()
        check(_lib().daspmm_server_stats(self._h, ctypes.byref(o)), "server_stats")
        return {n: getattr(o, n) for n, _ in o._fields_}

    def close(self):
        if self._h:
            _lib().daspmm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- problem
class SpmvSpmmProblem:
    """Non-owning view of device buffers with run/benchmark, after
    SpmvSpmmProblem (spmvspmm.h:13-50, 202-243).  `run` keeps the reference's
    power-of-two check and its print-and-return behaviour for bad nv."""

    def __init__(self, A: DeviceCsr, dnInput, dnOutput, maxNv: int):
        self.A, self.dnInput, self.dnOutput, self.maxNv = A, dnInput, dnOutput, maxNv

    def run(self, layout: int, nv: int, alg: int) -> None:
        if nv & (nv - 1):
            import sys
            print(f"nv must be power of 2, less than 32. Got nv = {nv}", file=sys.stderr)
            return
        err = compat_spmm(alg, layout, self.A, self.dnInput, self.dnOutput, nv)
        if err != 0:
            raise DaspmmError(3, f"cudaSpmm returned cudaError {err}")

    def benchmark(self, layout: int, nv: int, alg: int, warmupIters: int = 5,
                  repeatIters: int = 50) -> float:
        import torch
        if nv & (nv - 1):
            return -1.0
        for _ in range(warmupIters):
            compat_spmm(alg, layout, self.A, self.dnInput, self.dnOutput, nv)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(torch.cuda.default_stream())
        for _ in range(repeatIters):
            compat_spmm(alg, layout, self.A, self.dnInput, self.dnOutput, nv)
        e.record(torch.cuda.default_stream())
        e.synchronize()
        return s.elapsed_time(e) / repeatIters
