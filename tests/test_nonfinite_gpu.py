"""Inf / NaN in a row of B that A never references must not reach C.

The window kernels gather B rows in fixed windows of nonzeros and pad a
chunk's last window; a padded position must add nothing (0 * Inf is NaN).
Here column 0 of A is empty and row 0 of B (row-major; column 0 of each
column-major slice) holds Inf or NaN, so every element of the true product is
finite.  Every path -- the five algorithms in both layouts, the 16- and
32-lane window kernels over 32/64/128-column tiles, BF16 storage and the
batched kernel -- must return it (oracle rules of test_parity_gpu.py).
"""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALGS = [D.Alg.CSR_SCALAR, D.Alg.CSR_VECTOR, D.Alg.COO_SCALAR, D.Alg.COO_VECTOR,
        D.Alg.CSR_BALANCED]


def _shifted(A):
    """A with one empty column in front (column indices + 1)."""
    return D.Csr(A.nr, A.nc + 1, A.rowPtr.copy(), (A.colIdx + 1).astype(np.int32),
                 A.values.copy())


def _mats():
    return {"powerlaw": _shifted(D.gen_powerlaw(3000, dmax=400, seed=5)),
            "random": _shifted(D.gen_random(2000, 1500, 6.0, seed=6))}


def _b(A, nv, layout, bad, seed=1):
    B = np.random.default_rng(seed).uniform(-1, 1, A.nc * nv).astype(np.float32)
    if layout == D.Layout.ROW_MAJOR:
        B[:nv] = bad                       # B row 0: column 0 of A
    else:
        B[0::A.nc] = bad                   # element 0 of every column-major slice
    return B


def _check(A, layout, nv, B, C, what):
    assert np.isfinite(C).all(), f"{what}: non-finite values in C"
    ref = O.spmm_f32(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    ok, bad = O.check_result(layout, layout, A.nr, nv, ref, C, O.REF_ABS_TOL)
    assert ok, f"{what}: reference 1e-3 rule fails at {bad}"
    c64, absc = O.spmm_f64(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    assert O.rel_err(C, c64, absc) <= O.REL_TOL_F32, what


@pytest.mark.parametrize("bad", [np.inf, np.nan])
@pytest.mark.parametrize("layout", [D.Layout.ROW_MAJOR, D.Layout.COL_MAJOR])
def test_every_algorithm(cuda, bad, layout):
    import torch
    for name, A in _mats().items():
        dA = D.DeviceCsr(A)
        for nv in (1, 4, 32, 64, 128, 256):
            B = _b(A, nv, layout, bad)
            Bt = torch.from_numpy(B).cuda()
            for alg in ALGS:
                C = torch.full((A.nr * nv,), 7.0, device="cuda")
                D.spmm(alg, layout, dA, Bt, C, nv=nv)
                torch.cuda.synchronize()
                _check(A, layout, nv, B, C.cpu().numpy(), f"{name} alg {alg.name} nv {nv}")


@pytest.mark.parametrize("pipe", [1, 2, 3, 4])
def test_balanced_design_points(cuda, pipe):
    """CSR_BALANCED's register, TMA-ring, cp.async-ring and window pipes."""
    import torch
    for name, A in _mats().items():
        dA = D.DeviceCsr(A)
        for nv in (32, 64, 128):
            B = _b(A, nv, D.Layout.ROW_MAJOR, np.inf)
            Bt = torch.from_numpy(B).cuda()
            C = torch.full((A.nr * nv,), 7.0, device="cuda")
            D.spmm(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, dA, Bt, C, nv=nv,
                   cfg=D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=pipe))
            torch.cuda.synchronize()
            _check(A, D.Layout.ROW_MAJOR, nv, B, C.cpu().numpy(), f"{name} pipe {pipe} nv {nv}")


@pytest.mark.parametrize("bad", [np.inf, np.nan])
def test_32_lane_window_kernel_at_128_columns(cuda, bad):
    """B and C 16- but not 32-byte aligned: the 32-lane kernel takes N = 128."""
    import torch
    for name, A in _mats().items():
        dA = D.DeviceCsr(A)
        nv = 128
        B = _b(A, nv, D.Layout.ROW_MAJOR, bad)
        Bbuf = torch.zeros(A.nc * nv + 8, device="cuda")
        Cbuf = torch.zeros(A.nr * nv + 8, device="cuda")
        Bt, C = Bbuf[4:4 + A.nc * nv], Cbuf[4:4 + A.nr * nv]
        assert Bt.data_ptr() % 32 == 16 and C.data_ptr() % 32 == 16
        Bt.copy_(torch.from_numpy(B))
        D.spmm(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, dA, Bt, C, nv=nv)
        torch.cuda.synchronize()
        _check(A, D.Layout.ROW_MAJOR, nv, B, C.cpu().numpy(), f"{name} offset 16")


@pytest.mark.parametrize("nv", [64, 128])
def test_bf16_storage(cuda, nv):
    import torch
    for name, A in _mats().items():
        dA = D.DeviceCsr(A)
        B = _b(A, nv, D.Layout.ROW_MAJOR, np.inf)
        bq = D.quantize(torch.from_numpy(B).cuda(), D.Fmt.BF16)
        vq = D.quantize(dA.values, D.Fmt.BF16)
        C = torch.full((A.nr * nv,), 7.0, device="cuda")
        D.spmm_mixed(dA, vq, D.Fmt.BF16, bq, D.Fmt.BF16, C, nv)
        torch.cuda.synchronize()
        got = C.cpu().numpy()
        assert np.isfinite(got).all(), f"{name} nv {nv}: non-finite values in C"
        v64 = O.dequantize(1, vq.cpu().view(torch.int16).numpy().view(np.uint16))
        b64 = O.dequantize(1, bq.cpu().view(torch.int16).numpy().view(np.uint16))
        c64, absc = O.spmm_f64d(0, A.nr, A.nc, A.rowPtr, A.colIdx, v64, b64, nv)
        assert O.rel_err(got, c64, absc) <= O.REL_TOL_F32, f"{name} nv {nv}"


@pytest.mark.parametrize("bf", [D.Fmt.F32, D.Fmt.BF16])
@pytest.mark.parametrize("nv", [16, 64, 128])
def test_batched_kernel(cuda, nv, bf):
    import torch
    inst, hosts = [], []
    for name, A in _mats().items():
        for rep in range(2):
            dA = D.DeviceCsr(A)
            B = _b(A, nv, D.Layout.ROW_MAJOR, np.nan)
            Bt = torch.from_numpy(B).cuda()
            bq = Bt if bf == D.Fmt.F32 else D.quantize(Bt, bf)
            C = torch.full((A.nr * nv,), 7.0, device="cuda")
            inst.append(dict(A=dA, values=dA.values, val_fmt=D.Fmt.F32, B=bq, b_fmt=bf,
                             b_scales=None, C=C, nv=nv, beta=0.0))
            b64 = (B.astype(np.float64) if bf == D.Fmt.F32 else
                   O.dequantize(1, bq.cpu().view(torch.int16).numpy().view(np.uint16)))
            hosts.append((name, A, b64))
    b = D.Batch(inst, chunk=97)
    b.run()
    torch.cuda.synchronize()
    for d, (name, A, b64) in zip(inst, hosts):
        got = d["C"].cpu().numpy()
        assert np.isfinite(got).all(), f"{name} nv {nv}: non-finite values in C"
        c64, absc = O.spmm_f64d(0, A.nr, A.nc, A.rowPtr, A.colIdx,
                                A.values.astype(np.float64), b64, nv)
        assert O.rel_err(got, c64, absc) <= O.REL_TOL_F32, f"{name} nv {nv}"
    b.close()
