"""Python wrapper of the CPU oracle (liboracle.so) and, when built, of the
harness around the unmodified reference (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The product
(libdaspmm.so and its bindings) never imports this module.

Each function names the reference code it restates (see oracle.c).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref.so")

_VP = ctypes.c_void_p
_I = ctypes.c_int
_lib = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `make -C {HERE} oracle`")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "or_coo_to_csr_rowptr": (_I, [_I, _I, _VP, _VP]),
            "or_spmm_f32": (None, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP]),
            "or_spmm_f64": (None, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
            "or_spmm_f64d": (None, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
            "or_check_result": (_I, [_I, _I, _I, _I, _VP, _VP, ctypes.c_float, _I,
                                     ctypes.POINTER(_I), ctypes.POINTER(_I)]),
            "or_calc_max_nv": (_I, [_I, _I, _I, ctypes.c_size_t, _I, _I]),
            "or_row_of": (_I, [_VP, _I, _I]),
            "or_num_chunks": (_I, [_I, _I]),
            "or_balanced_partition": (None, [_I, _I, _VP, _I, _I, _VP]),
            "or_balanced_ownership": (_I, [_I, _I, _VP, _I, _I, _VP]),
            "or_coo_ownership": (_I, [_I, _I, _VP, _I, _VP]),
            "or_quantize": (None, [_I, ctypes.c_size_t, _VP, _VP]),
            "or_dequantize": (None, [_I, ctypes.c_size_t, _VP, _VP]),
            "or_gen_uniform": (_I, [_I, _I, _I, ctypes.c_uint64, _VP, _VP, _VP]),
            "or_gen_powerlaw": (_I, [_I, _I, ctypes.c_double, ctypes.c_double, _I, _I,
                                     ctypes.c_double, ctypes.c_uint64, _VP, _VP, _VP,
                                     ctypes.POINTER(ctypes.c_longlong)]),
            "or_gen_dense": (None, [ctypes.c_size_t, ctypes.c_uint64, ctypes.c_float,
                                    ctypes.c_float, _VP]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    """The unmodified reference's host code and kernels (oracle/_ref/libref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise ImportError(f"{REF_PATH} missing (built only where the reference tree exists)")
        R = ctypes.CDLL(REF_PATH)
        sig = {
            "ref_cpu_spmm": (None, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP]),
            "ref_coo_to_csr": (_I, [_I, _I, _VP, _VP]),
            "ref_check_result": (_I, [_I, _I, _I, _I, _VP, _VP, ctypes.c_float]),
            "ref_cpu_bench": (ctypes.c_double, [_I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _I, _I]),
            "ref_cuda_spmm": (_I, [_I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
            "ref_cuda_bench": (ctypes.c_float, [_I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP,
                                                _VP, _I, _I]),
            "ref_cusparse_bench": (ctypes.c_float, [_I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP,
                                                    _VP, _VP, _I, _I, _I]),
        }
        for n, (r, a) in sig.items():
            f = getattr(R, n)
            f.restype, f.argtypes = r, a
        _ref = R
    return _ref


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------- oracle
def coo_to_csr(nr: int, rowIdx) -> np.ndarray:
    """generateCsrRowPtrArray (spmvspmm_benchmark.cu:41-76)."""
    ri = _i32(rowIdx)
    rp = np.zeros(nr + 1, np.int32)
    if lib().or_coo_to_csr_rowptr(nr, ri.size, _p(ri), _p(rp)) != 0:
        raise ValueError("rowIdx not sorted or out of range")
    return rp


def spmm_f32(layout: int, nr: int, nc: int, rowPtr, colIdx, values, B, nv: int) -> np.ndarray:
    """cpuSpmvReference (spmvspmm_benchmark.cu:11-39); returns C flat in `layout`."""
    rp, ci, va, b = _i32(rowPtr), _i32(colIdx), _f32(values), _f32(B).reshape(-1)
    C = np.zeros(nr * nv, np.float32)
    lib().or_spmm_f32(int(layout), nr, nc, int(rp[-1]) if nr else 0, nv, _p(rp), _p(ci), _p(va),
                      _p(b), _p(C))
    return C


def spmm_f64(layout: int, nr: int, nc: int, rowPtr, colIdx, values, B, nv: int):
    """FP64 product and the condition scale sum|a||b| per output element."""
    rp, ci, va, b = _i32(rowPtr), _i32(colIdx), _f32(values), _f32(B).reshape(-1)
    C = np.zeros(nr * nv, np.float64)
    A = np.zeros(nr * nv, np.float64)
    lib().or_spmm_f64(int(layout), nr, nc, int(rp[-1]) if nr else 0, nv, _p(rp), _p(ci), _p(va),
                      _p(b), _p(C), _p(A))
    return C, A


def spmm_f64d(layout: int, nr: int, nc: int, rowPtr, colIdx, values64, B64, nv: int):
    rp, ci = _i32(rowPtr), _i32(colIdx)
    va = np.ascontiguousarray(values64, np.float64)
    b = np.ascontiguousarray(B64, np.float64).reshape(-1)
    C = np.zeros(nr * nv, np.float64)
    A = np.zeros(nr * nv, np.float64)
    lib().or_spmm_f64d(int(layout), nr, nc, int(rp[-1]) if nr else 0, nv, _p(rp), _p(ci), _p(va),
                       _p(b), _p(C), _p(A))
    return C, A


def check_result(host_layout: int, dev_layout: int, nrows: int, ncols: int, ref, out,
                 eps: float = 1e-3, first_only: bool = True):
    """checkResult (spmvspmm_benchmark.cu:93-116): (passed, first_bad_(i, j))."""
    r, o = _f32(ref), _f32(out)
    bi, bj = _I(-1), _I(-1)
    ok = lib().or_check_result(host_layout, dev_layout, nrows, ncols, _p(r), _p(o), eps,
                               int(first_only), ctypes.byref(bi), ctypes.byref(bj))
    return bool(ok), (bi.value, bj.value)


def calc_max_nv(nr: int, nc: int, nnz: int, mem_bytes: int, dtype_size: int = 4,
                maxnv: int = 128) -> int:
    """calcMaxNv (spmvspmm_benchmark.cu:78-90)."""
    return lib().or_calc_max_nv(nr, nc, nnz, mem_bytes, dtype_size, maxnv)


def num_chunks(nnz: int, chunk: int) -> int:
    return lib().or_num_chunks(nnz, chunk)


def balanced_partition(nr: int, rowPtr, chunk: int, snap: int) -> np.ndarray:
    rp = _i32(rowPtr)
    n = num_chunks(int(rp[-1]), chunk)
    meta = np.zeros(2 * (n + 1), np.int32)
    lib().or_balanced_partition(nr, int(rp[-1]), _p(rp), chunk, snap, _p(meta))
    return meta


def balanced_ownership(nr: int, rowPtr, chunk: int, snap: int) -> np.ndarray:
    rp = _i32(rowPtr)
    own = np.zeros(2 * max(1, nr), np.int32)
    if lib().or_balanced_ownership(nr, int(rp[-1]), _p(rp), chunk, snap, _p(own)) != 0:
        raise AssertionError("balanced ownership walk inconsistent")
    return own[: 2 * nr]


def coo_ownership(nr: int, rowIdx, chunk: int) -> np.ndarray:
    ri = _i32(rowIdx)
    own = np.zeros(2 * max(1, nr), np.int32)
    if lib().or_coo_ownership(nr, ri.size, _p(ri), chunk, _p(own)) != 0:
        raise AssertionError("COO ownership walk inconsistent")
    return own[: 2 * nr]


_QDT = {0: np.float32, 1: np.uint16, 2: np.uint16, 3: np.uint8}


def quantize(fmt: int, x) -> np.ndarray:
    """Round float32 values to BF16 / FP16 / FP8-E4M3 storage (nearest even)."""
    xf = _f32(x).reshape(-1)
    q = np.zeros(xf.size, _QDT[fmt])
    lib().or_quantize(fmt, xf.size, _p(xf), _p(q))
    return q


def dequantize(fmt: int, q) -> np.ndarray:
    q = np.ascontiguousarray(q, _QDT[fmt]).reshape(-1)
    x = np.zeros(q.size, np.float64)
    lib().or_dequantize(fmt, q.size, _p(q), _p(x))
    return x


# ---------------------------------------------------------------- workloads
class HostCsr:
    """A host CSR matrix built by the oracle's generators (int32 / float32)."""

    def __init__(self, nr, nc, rowPtr, colIdx, values):
        self.nr, self.nc = nr, nc
        self.rowPtr, self.colIdx, self.values = rowPtr, colIdx, values

    @property
    def nnz(self) -> int:
        return int(self.rowPtr[-1]) if self.nr > 0 else 0

    def cols_touched(self) -> int:
        return int(np.unique(self.colIdx).size) if self.nnz else 0


def gen_uniform(nr: int, nc: int, per_row: int, seed: int = 0) -> HostCsr:
    """Exactly per_row distinct uniform columns per row, values U(-1,1)
    (restates libdaspmm's daspmm_gen_uniform)."""
    rp = np.zeros(nr + 1, np.int32)
    n = nr * per_row
    ci = np.zeros(max(1, n), np.int32)
    va = np.zeros(max(1, n), np.float32)
    if lib().or_gen_uniform(nr, nc, per_row, seed, _p(rp), _p(ci), _p(va)) != 0:
        raise ValueError("gen_uniform: bad arguments")
    return HostCsr(nr, nc, rp, ci[:n].copy(), va[:n].copy())


def gen_powerlaw(n: int, alpha: float = 2.1, shift: float = 0.16, dmin: int = 1,
                 dmax: int = 4096, seed: int = 0, mean_scale: float = 1.0,
                 nc: int | None = None) -> HostCsr:
    """Power-law out-degrees (k + shift)^-alpha on [dmin, dmax], preferential-
    attachment columns, values U(-1,1) (restates daspmm_gen_powerlaw)."""
    nc = n if nc is None else nc
    rp = np.zeros(n + 1, np.int32)
    nnz = ctypes.c_longlong(0)
    if lib().or_gen_powerlaw(n, nc, alpha, shift, dmin, dmax, mean_scale, seed, _p(rp), None,
                             None, ctypes.byref(nnz)) != 0:
        raise ValueError("gen_powerlaw: bad arguments")
    ci = np.zeros(max(1, nnz.value), np.int32)
    va = np.zeros(max(1, nnz.value), np.float32)
    lib().or_gen_powerlaw(n, nc, alpha, shift, dmin, dmax, mean_scale, seed, _p(rp), _p(ci),
                          _p(va), ctypes.byref(nnz))
    return HostCsr(n, nc, rp, ci[:nnz.value].copy(), va[:nnz.value].copy())


def gen_dense(n: int, seed: int = 1, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    """n floats U(lo, hi) on a 2^-24 grid (restates daspmm_gen_dense)."""
    out = np.empty(max(1, n), np.float32)
    lib().or_gen_dense(n, seed, lo, hi, _p(out))
    return out[:n]


# ---------------------------------------------------------------- tolerances
# FP32 parity rule, stated once for every test:
#   (1) the reference's own check: |gpu - host_fp32| <= 1e-3 absolute
#       (checkResult, spmvspmm_benchmark.cu:94,103);
#   (2) against FP64: |gpu - c64| <= REL_TOL_F32 * sum_p |a_p||b_p| + 1e-30,
#       i.e. relative to the condition scale of each element.  A recursive
#       FP32 sum of n products has error <= n*u*sum|a||b| (u = 2^-24); the
#       kernels' sums are shorter chains (per lane, then a tree), and for the
#       rows here (<= 4096 nonzeros) 2e-5 covers the serial host loop too.
REF_ABS_TOL = 1e-3
REL_TOL_F32 = 2e-5


# Mixed precision (storage in BF16 / FP16 / E4M3, FP32 arithmetic): the error
# statement is max |c - c64| / max sum_p |a_p||b_p| over the whole result (a
# max-norm relative error).  A per-element bound cannot hold for reduced
# storage: a one-term output whose operand rounds to a subnormal or to zero is
# off by up to 100% of itself.  Bounds: BF16 / FP16 storage <= 1e-2 (rounding
# 2^-9 / 2^-12 per operand); E4M3 B <= 2^-4 (3-bit mantissa, rounding 2^-4).
MIXED_TOL = 1e-2
E4M3_TOL = 2.0 ** -4


def rel_err_max(c, c64, absc) -> float:
    """max |c - c64| / max sum|a||b| (0 for an all-zero product)."""
    c = np.asarray(c, np.float64).reshape(-1)
    m = float(np.max(absc)) if np.size(absc) else 0.0
    d = float(np.max(np.abs(c - c64))) if c.size else 0.0
    return d / m if m > 0 else (0.0 if d == 0 else float("inf"))


def rel_err(c, c64, absc) -> float:
    """max |c - c64| / sum|a||b| over all elements (0 where the scale is 0)."""
    c = np.asarray(c, np.float64).reshape(-1)
    d = np.abs(c - c64)
    scale = np.where(absc > 0, absc, 1.0)
    bad = (absc == 0) & (d > 0)
    if bad.any():
        return float("inf")
    return float((d / scale).max()) if d.size else 0.0


def row_slice(rowPtr, colIdx, values, r0: int, r1: int):
    """Rows [r0, r1) of a CSR matrix with their columns renumbered 0..m-1:
    (rowPtr, colIdx, values, cols), where cols[j] is the original column of
    new column j.  Lets the FP64 oracle check a row sample of a large product
    with only the B rows that sample reads."""
    rp = np.asarray(rowPtr)
    p0, p1 = int(rp[r0]), int(rp[r1])
    ci = np.asarray(colIdx[p0:p1])
    cols = np.unique(ci)
    return ((rp[r0:r1 + 1] - p0).astype(np.int32), np.searchsorted(cols, ci).astype(np.int32),
            np.ascontiguousarray(values[p0:p1]), cols)


ERR_FLOOR = 1e-3


def error_stats(c, c64, absc) -> dict:
    """Three statements of |c - c64| (c64 the FP64 oracle, absc = sum|a||b|
    per element), over every element given:
      norm_max      max|c - c64| / max absc            (max-norm relative)
      cond_max      max |c - c64| / absc               (per element, relative to
                                                        its own condition scale)
      rel_floored   max |c - c64| / max(|c64|, ERR_FLOOR * max|c64|)
                                                       (per element, relative to
                                                        itself, small values floored)"""
    c = np.asarray(c, np.float64).reshape(-1)
    d = np.abs(c - c64)
    m64 = float(np.max(np.abs(c64))) if c64.size else 0.0
    den = np.maximum(np.abs(c64), ERR_FLOOR * m64) if m64 > 0 else np.ones_like(c64)
    return {"norm_max": rel_err_max(c, c64, absc), "cond_max": rel_err(c, c64, absc),
            "rel_floored": float((d / den).max()) if d.size else 0.0}


def sample_rows(rowPtr, colIdx, nv: int, cap: int = 1 << 25) -> int:
    """How many leading rows the FP64 oracle checks for an nv-column product:
    all of them when the sample's output and its B rows stay under `cap`
    elements each, else the largest power-of-two row count that does."""
    rp = np.asarray(rowPtr)
    nr = rp.size - 1
    R = min(nr, max(1, cap // nv))
    while R > 1:
        ncols = np.unique(np.asarray(colIdx[: int(rp[R])])).size
        if ncols * nv <= cap:
            break
        R //= 2
    return R


def mixed_errors(rp, ci, va32, va64, b32, b64, c, nv: int) -> dict:
    """Error statements of a mixed-precision product on a row sample
    (row_slice's compacted form): va32 / b32 the original FP32 values and B
    rows, va64 / b64 their stored (quantized, scales applied) values as FP64,
    c the device result for those rows.  `kernel` is the kernel's own
    arithmetic (against FP64 of the stored inputs, per element relative to
    its condition scale); `storage` is storage + arithmetic (against FP64 of
    the FP32 inputs), as error_stats."""
    nr, nc = rp.size - 1, b32.size // nv
    cq, aq = spmm_f64d(0, nr, nc, rp, ci, va64, b64, nv)
    c64, a64 = spmm_f64(0, nr, nc, rp, ci, va32, b32, nv)
    return {"kernel": rel_err(c, cq, aq), "storage": error_stats(c, c64, a64)}


def read_mtx(path: str, keep_diagonal: bool = False):
    """readMtx<float> (util/spmatrix.hpp:286-333) restated for small files,
    with makeSymmetric's value alignment fixed: returns (nr, nc, rows, cols,
    vals) sorted by (row, col, position in the file).  A symmetric file is
    mirrored (spmatrix.hpp:225-232) and loses diagonal entries and repeated
    (row, col) pairs (:244-263); pattern entries have value 1 (:166-180)."""
    with open(path) as f:
        lines = f.read().split("\n")
    banner = lines[0].lower().split()
    field, sym = banner[3], banner[4]
    i = 1
    while not lines[i].strip() or lines[i].lstrip().startswith("%"):
        i += 1
    nr, nc, nz = (int(x) for x in lines[i].split()[:3])
    ent = []
    for k, line in enumerate(lines[i + 1: i + 1 + nz]):
        t = line.split()
        v = 1.0 if field == "pattern" else float(np.float32(float(t[2])))
        ent.append((int(t[0]) - 1, int(t[1]) - 1, k, v))
    if sym == "symmetric":
        ent += [(c, r, nz + k, v) for (r, c, k, v) in ent if r != c]
    ent.sort(key=lambda e: (e[0], e[1], e[2]))
    if sym == "symmetric":
        kept = []
        for e in ent:
            if e[0] == e[1] and not keep_diagonal:
                continue
            if kept and kept[-1][0] == e[0] and kept[-1][1] == e[1]:
                continue
            kept.append(e)
        ent = kept
    rows = np.array([e[0] for e in ent], np.int32)
    cols = np.array([e[1] for e in ent], np.int32)
    vals = np.array([e[3] for e in ent], np.float32)
    return nr, nc, rows, cols, vals
