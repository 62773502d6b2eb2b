"""The drop-in layer on the GPU.

1. The reference's UNMODIFIED benchmark driver (spmvspmm_benchmark.cu),
   compiled against include/spmvspmm.h etc. and linked with libdaspmm.so
   (oracle/_ref/spmvspmm_compat, built by oracle/Makefile), reads a Matrix
   Market file and runs its own checkAlgorithms: every algorithm x layout x
   nv = 1..128 against its host loop at 1e-3 (spmvspmm_benchmark.cu:118-233),
   plus cuSPARSE.  It exits 0 only if all pass, then prints its CSV rows.
2. The kernel templates of include/spmm.h / spmv.h launched with the
   reference dispatcher's own grids give the oracle's product.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "spmvspmm_compat")
TEMPLATES = os.path.join(ROOT, "tests", "compat", "liblaunch_templates.so")


def write_mtx(path, A):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.nr} {A.nc} {A.nnz}\n")
        rows = A.rowIdx + 1
        cols = A.colIdx + 1
        for r, c, v in zip(rows.tolist(), cols.tolist(), A.values.tolist()):
            f.write(f"{r} {c} {v:.9g}\n")


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="compat driver not built")
@pytest.mark.parametrize("kind", ["powerlaw", "uniform"])
def test_reference_driver_checks_pass(cuda, tmp_path, kind):
    A = (D.gen_powerlaw(20000, dmax=2000, seed=2) if kind == "powerlaw"
         else D.gen_uniform(4096, 4096, 16, seed=0))
    mtx = tmp_path / f"{kind}.mtx"
    write_mtx(mtx, A)
    p = subprocess.run([DRIVER, str(mtx)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, f"reference checkAlgorithms failed:\n{p.stderr[-3000:]}"
    assert "Check Failed" not in p.stderr
    rows = [ln for ln in p.stdout.splitlines() if ln.startswith(str(mtx))]
    # one CSV row per nv = 1, 2, 4, ..., 128: filename, nv, 8 own variants, cuSPARSE columns
    assert [int(r.split(",")[1]) for r in rows] == [1, 2, 4, 8, 16, 32, 64, 128]
    for r in rows:
        own = [float(x) for x in r.split(",")[2:10]]
        assert all(x > 0 for x in own), r
    with open(os.path.join(str(tmp_path), "driver_stdout.csv"), "w") as f:
        f.write(p.stdout)


@pytest.mark.skipif(not os.path.exists(TEMPLATES), reason="template harness not built")
def test_templates_under_reference_grids(cuda):
    import torch
    lib = ctypes.CDLL(TEMPLATES)
    f = lib.launch_ref_grid
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p] * 6
    A = D.gen_powerlaw(6000, dmax=900, seed=4)
    dA = D.DeviceCsr(A)
    rng = np.random.default_rng(1)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for nv in (1, 2, 4, 8, 16, 32, 64, 128):
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        Bt = torch.from_numpy(B).cuda()
        for layout in (0, 1):
            ref = O.spmm_f32(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
            for alg in (0, 1, 2, 3):
                Ct = torch.zeros(A.nr * nv, dtype=torch.float32, device="cuda")
                err = f(alg, layout, A.nr, A.nc, A.nnz, nv, p(dA.rowPtr), p(dA.rowIdx),
                        p(dA.colIdx), p(dA.values), p(Bt), p(Ct))
                assert err == 0, (alg, layout, nv, err)
                torch.cuda.synchronize()
                ok, bad = O.check_result(layout, layout, A.nr, nv, ref, Ct.cpu().numpy())
                assert ok, (alg, layout, nv, bad)
