"""The reference's own GPU kernels on B200, against this library.

oracle/_ref/libref.so is the unmodified reference (spmvspmm.h, spmm.h,
spmv.h) compiled for sm_100a; ref_cuda_spmm is its dispatcher cudaSpmm<256,32>
(spmvspmm.h:53-199).  For the four algorithms x two layouts of the
reference's benchmark (spmvspmm_benchmark.cu:289-296) and N in {1, 32, 128},
daspmm_spmm's result must agree with the reference kernels' result under the
reference's own check (|a - b| <= 1e-3, checkResult, spmvspmm_benchmark.cu:
93-116), and both must be within the FP64 rule of every parity test
(|c - c64| <= 2e-5 * sum|a||b|).  Every launch here has a grid of at least
one block (the reference's vector dispatch floors numberOfWarps / 8, which is
zero below 8 warps, spmvspmm.h:122): the matrices are sized so it never is.
Skipped where the reference tree was not present to build libref.so.
"""
import ctypes

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_VP = ctypes.c_void_p


def _p(t):
    return _VP(t.data_ptr())


@pytest.fixture(scope="module")
def ref(cuda):
    if not O.ref_available():
        pytest.skip("oracle/_ref/libref.so not built (no reference tree where it was built)")
    return O.ref()


@pytest.mark.parametrize("which", ["powerlaw", "uniform"])
def test_reference_kernels_agree(ref, which):
    import torch
    A = (D.gen_powerlaw(20000, dmax=2000, seed=8) if which == "powerlaw"
         else D.gen_uniform(4096, 4096, 16, seed=0))
    dA = D.DeviceCsr(A)
    # the reference's vector dispatch: min(ceil(nnz/32), nr) * columns/4 warps, / 8 per block
    assert min((A.nnz + 31) // 32, A.nr) >= 8
    rng = np.random.default_rng(3)
    for nv in (1, 32, 128):
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        Bt = torch.from_numpy(B).cuda()
        for layout in (0, 1):
            c64, absc = O.spmm_f64(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
            for alg in range(4):
                Cr = torch.zeros(A.nr * nv, device="cuda")   # COO kernels accumulate
                st = ref.ref_cuda_spmm(alg, layout, A.nr, A.nc, A.nnz, nv, _p(dA.rowPtr),
                                       _p(dA.rowIdx), _p(dA.colIdx), _p(dA.values), _p(Bt),
                                       _p(Cr))
                torch.cuda.synchronize()
                assert st == 0, f"reference launch failed: cudaError {st}"
                Co = torch.full((A.nr * nv,), float("nan"), device="cuda")
                D.spmm(alg, layout, dA, Bt, Co, nv=nv)
                torch.cuda.synchronize()
                cr, co = Cr.cpu().numpy(), Co.cpu().numpy()
                what = f"{which} nv={nv} layout={layout} alg={alg}"
                ok, bad = O.check_result(layout, layout, A.nr, nv, cr, co, O.REF_ABS_TOL)
                assert ok, f"{what}: differs from the reference kernel at {bad}"
                assert O.rel_err(co, c64, absc) <= O.REL_TOL_F32, what
                assert O.rel_err(cr, c64, absc) <= O.REL_TOL_F32, f"{what} (reference kernel)"
