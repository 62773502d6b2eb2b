"""The bounded shared-memory barrier wait of the ring kernels runs out and
reports, without a fault or a hang.

daspmm_wait_probe arms a barrier for transaction bytes that no copy will ever
deliver (nothing is issued, so nothing is in flight when the kernel leaves)
and waits on it with the same mbar_wait the TMA / cp.async rings use, under a
short poll bound.  The kernel must return, daspmm_device_error() must report
DASPMM_ERR_TIMEOUT once (and then be clear), and the context must stay
usable: a normal SpMM right after it matches the oracle."""
import ctypes

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DASPMM_ERR_TIMEOUT = 6


def test_wait_runs_out_and_reports(cuda):
    import torch
    L = D.lib()
    assert L.daspmm_device_error() == 0          # clear any earlier state
    out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    # a wait that completes: no error
    D.check(L.daspmm_wait_probe(64, 0, ctypes.c_void_p(out.data_ptr()), None), "wait_probe")
    torch.cuda.synchronize()
    assert int(out.item()) == 1
    assert L.daspmm_device_error() == 0
    # a wait on bytes nothing delivers: runs out, reports, kernel returns
    for polls in (1, 1000):
        out.fill_(-1)
        D.check(L.daspmm_wait_probe(polls, 1, ctypes.c_void_p(out.data_ptr()), None),
                "wait_probe")
        torch.cuda.synchronize()
        assert int(out.item()) == 0
        assert L.daspmm_device_error() == DASPMM_ERR_TIMEOUT
        assert L.daspmm_device_error() == 0      # read clears it
    # the context is still usable
    A = D.gen_powerlaw(2000, dmax=200, seed=4)
    dA = D.DeviceCsr(A)
    nv = 32
    B = D.gen_dense(A.nc * nv, seed=2)
    C = torch.zeros(A.nr * nv, device="cuda")
    cfg = D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=2)     # the TMA ring itself
    D.spmm(D.Alg.CSR_BALANCED, 0, dA, torch.from_numpy(B).cuda(), C, nv=nv, cfg=cfg)
    torch.cuda.synchronize()
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    ok, bad = O.check_result(0, 0, A.nr, nv, ref, C.cpu().numpy(), O.REF_ABS_TOL)
    assert ok, bad
    assert L.daspmm_device_error() == 0


def test_wait_probe_rejects_bad_arguments(cuda):
    L = D.lib()
    assert L.daspmm_wait_probe(0, 1, ctypes.c_void_p(8), None) != 0
    assert L.daspmm_wait_probe(10, 1, None, None) != 0
