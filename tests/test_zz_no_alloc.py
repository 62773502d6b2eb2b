"""daspmm_spmm_noalloc: the SpMM entry point for callers that cannot allocate.

A plugin whose host application owns all device memory, or a loop that must
not synchronise the device through cudaMalloc/cudaFree, cannot use
daspmm_spmm (it allocates its workspace on first use).  daspmm_spmm_noalloc
runs the same balanced-CSR kernels with scratch taken from a fixed array
inside the library.  These tests call it through the C ABI (ctypes), twice in
a row, and compare it with daspmm_spmm on the same inputs, under the same
tolerances as every other parity test (oracle/oracle.py).  The file is named
so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_VP = ctypes.c_void_p


def _noalloc():
    f = D.lib().daspmm_spmm_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 5 + [_VP] * 5 + [ctypes.c_float, _VP]
    return f


def _p(t):
    return _VP(t.data_ptr())


def _both(A, dA, layout, nv, B, beta=0.0, C0=None):
    """(noalloc result, daspmm_spmm result) for the same inputs."""
    import torch
    Bt = torch.from_numpy(B).cuda()
    init = (torch.from_numpy(C0).cuda() if C0 is not None
            else torch.zeros(A.nr * nv, dtype=torch.float32, device="cuda"))
    Cn = init.clone()
    Ce = init.clone()
    st = _noalloc()(layout, A.nr, A.nc, A.nnz, nv, _p(dA.rowPtr), _p(dA.colIdx),
                    _p(dA.values), _p(Bt), _p(Cn), beta, None)
    assert st == 0, D.lib().daspmm_status_string(st)
    D.spmm(D.Alg.CSR_BALANCED, layout, dA, Bt, Ce, beta=beta, nv=nv)
    torch.cuda.synchronize()
    return Cn.cpu().numpy(), Ce.cpu().numpy()


def _agree(A, layout, nv, B, Cn, Ce, beta=0.0, C0=None):
    ok, bad = O.check_result(layout, layout, A.nr, nv, Ce, Cn, O.REF_ABS_TOL)
    assert ok, f"noalloc vs daspmm_spmm differ at {bad}"
    c64, absc = O.spmm_f64(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    if beta != 0.0:
        c64 = c64 + beta * C0.astype(np.float64)
        absc = absc + abs(beta) * np.abs(C0.astype(np.float64))
    assert O.rel_err(Cn, c64, absc) <= O.REL_TOL_F32


def test_two_calls_in_a_row_match_existing_entry_point(cuda):
    rng = np.random.default_rng(21)
    A = D.gen_powerlaw(30000, dmax=3000, seed=7)      # hub rows split across chunks
    dA = D.DeviceCsr(A)
    for layout, nv in ((0, 128), (0, 32)):
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        for _ in range(2):                           # second call sees the first's leftovers
            Cn, Ce = _both(A, dA, layout, nv, B)
            _agree(A, layout, nv, B, Cn, Ce)
    # a smaller problem right after a larger one, and col-major with beta
    S = D.gen_uniform(500, 400, 9, seed=3)
    dS = D.DeviceCsr(S)
    B = rng.uniform(-1, 1, S.nc * 16).astype(np.float32)
    C0 = rng.uniform(-1, 1, S.nr * 16).astype(np.float32)
    for _ in range(2):
        Cn, Ce = _both(S, dS, 1, 16, B, beta=0.5, C0=C0)
        _agree(S, 1, 16, B, Cn, Ce, beta=0.5, C0=C0)


def test_full_size_power_law_fits_and_matches(cuda):
    """The 262,144-row power-law matrix at N = 128 fits the fixed scratch."""
    A = D.gen_powerlaw(262144, seed=0)
    dA = D.DeviceCsr(A)
    B = D.gen_dense(A.nc * 128, seed=1)
    cfg = D.default_config(D.Alg.CSR_BALANCED, 0, A.nr, A.nc, A.nnz, 128)
    assert D.workspace_bytes(cfg, 0, A.nr, A.nc, A.nnz, 128) <= (16 << 20)
    for _ in range(2):
        Cn, Ce = _both(A, dA, 0, 128, B)
        ok, bad = O.check_result(0, 0, A.nr, 128, Ce, Cn, O.REF_ABS_TOL)
        assert ok, bad


def test_too_large_is_refused_before_device_work(cuda):
    import torch
    # one chunk per resident warp x 4096 columns x 8 bytes: far over the 16 MiB limit
    nr = 1 << 20
    nnz = 2_200_000
    nv = 4096
    cfg = D.default_config(D.Alg.CSR_BALANCED, 0, nr, nr, nnz, nv)
    assert D.workspace_bytes(cfg, 0, nr, nr, nnz, nv) > (16 << 20)
    dummy = torch.zeros(4, dtype=torch.float32, device="cuda")
    st = _noalloc()(0, nr, nr, nnz, nv, _p(dummy), _p(dummy), _p(dummy), _p(dummy), _p(dummy),
                    0.0, None)
    assert st == 5   # DASPMM_ERR_WORKSPACE
    torch.cuda.synchronize()


def test_column_major_limit(cuda):
    """Column-major calls gather B directly (no room for copies of B and C), so
    their limit is the workspace of {CSR_BALANCED, pipe 1}: the largest nv
    under the limit runs and matches daspmm_spmm, the next one is refused."""
    import torch
    A = D.gen_random(200000, 200000, 8.0, seed=4)
    dA = D.DeviceCsr(A)
    cfg = D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=1)
    ws = lambda nv: D.workspace_bytes(cfg, 1, A.nr, A.nc, A.nnz, nv)
    fit = max(nv for nv in range(1, 200) if ws(nv) <= (16 << 20))
    assert ws(fit + 1) > (16 << 20)
    rng = np.random.default_rng(5)
    B = rng.uniform(-1, 1, A.nc * fit).astype(np.float32)
    for _ in range(2):
        Cn, Ce = _both(A, dA, 1, fit, B)
        _agree(A, 1, fit, B, Cn, Ce)
    Bt = torch.zeros(A.nc * (fit + 1), device="cuda")
    C = torch.zeros(A.nr * (fit + 1), device="cuda")
    st = _noalloc()(1, A.nr, A.nc, A.nnz, fit + 1, _p(dA.rowPtr), _p(dA.colIdx),
                    _p(dA.values), _p(Bt), _p(C), 0.0, None)
    assert st == 5   # DASPMM_ERR_WORKSPACE
    torch.cuda.synchronize()
