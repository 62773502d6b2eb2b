"""The benchmark's reference arm builds its inputs with the oracle's
restatement of the library's seeded generators, so that arm never loads the
product library.  These restatements must give the library's matrices and
dense operands bit for bit, at the benchmark's full size too."""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O


def _same(a, b):
    assert a.nr == b.nr and a.nc == b.nc
    np.testing.assert_array_equal(a.rowPtr, b.rowPtr)
    np.testing.assert_array_equal(a.colIdx, b.colIdx)
    assert a.values.dtype == b.values.dtype == np.float32
    np.testing.assert_array_equal(a.values.view(np.uint32), b.values.view(np.uint32))


@pytest.mark.parametrize("n,dmax,seed,scale", [(1, 4096, 0, 1.0), (97, 50, 3, 1.0),
                                               (4096, 300, 7, 2.5), (20000, 4096, 1, 0.5)])
def test_powerlaw_matches_library(n, dmax, seed, scale):
    _same(O.gen_powerlaw(n, dmax=dmax, seed=seed, mean_scale=scale),
          D.gen_powerlaw(n, dmax=dmax, seed=seed, mean_scale=scale))


def test_powerlaw_rectangular_matches_library():
    _same(O.gen_powerlaw(3000, dmax=900, seed=5, nc=1000),
          D.gen_powerlaw(3000, dmax=900, seed=5, nc=1000))


@pytest.mark.parametrize("nr,nc,k,seed", [(4096, 4096, 16, 0), (100, 17, 17, 2), (5, 9, 0, 1)])
def test_uniform_matches_library(nr, nc, k, seed):
    _same(O.gen_uniform(nr, nc, k, seed), D.gen_uniform(nr, nc, k, seed))


@pytest.mark.parametrize("n,seed,lo,hi", [(0, 1, -1.0, 1.0), (12345, 1, -1.0, 1.0),
                                          (777, 9, -0.5, 2.0)])
def test_dense_matches_library(n, seed, lo, hi):
    a = O.gen_dense(n, seed, lo, hi)
    b = D.gen_dense(n, seed, lo, hi)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_benchmark_inputs_match_library_full_size():
    # the FP32 headline workload: 262,144-row power-law graph (seed 0) and the
    # 262,144 x 128 dense operand (seed 1)
    _same(O.gen_powerlaw(262144, seed=0), D.gen_powerlaw(262144, seed=0))
    n = 262144 * 128
    np.testing.assert_array_equal(O.gen_dense(n, 1).view(np.uint32),
                                  D.gen_dense(n, 1).view(np.uint32))


def test_bad_arguments_rejected():
    with pytest.raises(ValueError):
        O.gen_powerlaw(10, dmin=5, dmax=2)
    with pytest.raises(ValueError):
        O.gen_uniform(4, 3, 4)
