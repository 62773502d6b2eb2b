"""Host-buffer entry points (daspmm_spmm_host, daspmm_spmm_host_async).

A, B and C live in host memory; the library copies them to its device
staging, runs the SpMM and copies C back.  Results follow the reference's
checkResult rule against the oracle; beta != 0 reads C from the host.
"""
import ctypes

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_p = lambda a: ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _call(fn, alg, A, B, C, nv, beta, stream=None, pinned=None):
    cfg = D.default_config(alg, 0, A.nr, A.nc, A.nnz, nv)
    rp = A.rowPtr
    ri = A.rowIdx if alg in (D.Alg.COO_SCALAR, D.Alg.COO_VECTOR) else None
    st = fn(ctypes.byref(cfg), 0, A.nr, A.nc, A.nnz, nv, _p(rp), _p(ri), _p(A.colIdx),
            _p(A.values), _p(B), _p(C), float(beta), stream)
    D.check(st, fn.__name__)


@pytest.mark.parametrize("alg", [D.Alg.CSR_SCALAR, D.Alg.CSR_VECTOR, D.Alg.COO_SCALAR,
                                 D.Alg.CSR_BALANCED])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_host_entry_matches_oracle(cuda, alg, beta):
    A = D.gen_powerlaw(6000, dmax=500, seed=3)
    nv = 64
    B = D.gen_dense(A.nc * nv, seed=4)
    C0 = D.gen_dense(A.nr * nv, seed=5)
    C = C0.copy()
    _call(D.lib().daspmm_spmm_host, alg, A, B, C, nv, beta)
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    ref = ref + np.float32(beta) * C0                 # every algorithm: C = A*B + beta*C
    assert O.check_result(0, 0, A.nr, nv, ref, C)[0]


def test_host_async_two_streams(cuda):
    import torch
    A = D.gen_powerlaw(20000, seed=7)
    nv = 128
    B = D.gen_dense(A.nc * nv, seed=8)
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    pin = lambda a: torch.from_numpy(a).pin_memory()
    rp, ci, va, Bh = pin(A.rowPtr), pin(A.colIdx), pin(A.values), pin(B)
    Cs = [torch.zeros(A.nr * nv).pin_memory() for _ in range(2)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    cfg = D.default_config(D.Alg.CSR_BALANCED, 0, A.nr, A.nc, A.nnz, nv)
    f = D.lib().daspmm_spmm_host_async
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    for i in range(6):
        D.check(f(ctypes.byref(cfg), 0, A.nr, A.nc, A.nnz, nv, vp(rp), None, vp(ci), vp(va),
                  vp(Bh), vp(Cs[i % 2]), 0.0, ctypes.c_void_p(streams[i % 2].cuda_stream)),
                "spmm_host_async")
    torch.cuda.synchronize()
    for c in Cs:
        assert O.check_result(0, 0, A.nr, nv, ref, c.numpy())[0]
    assert np.array_equal(Cs[0].numpy(), Cs[1].numpy())
