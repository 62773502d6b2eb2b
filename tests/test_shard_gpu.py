"""Row shards on the GPU: each rank's part computed by the library.

Only one GPU is available to the tests, so the ranks' parts are computed one
after another on cuda:0 (no rank waits on another: the sharded path has no
exchange).  The concatenated parts must satisfy the reference's check
against the oracle's product of the whole matrix.
"""
import numpy as np
import pytest

import daspmm as D
from daspmm import shard as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 4, 8])
def test_row_sharded_spmm(cuda, world):
    import torch
    A = D.gen_powerlaw(40000, seed=5)
    nv = 128
    B = torch.from_numpy(D.gen_dense(A.nc * nv, seed=6)).cuda()
    parts = []
    for rank in range(world):
        R = S.RowShardedSpmm(A, rank, world, device="cuda")
        C = torch.empty(R.local.nr * nv, device="cuda")
        R.spmm(B, C, nv)
        parts.append(C)
    torch.cuda.synchronize()
    got = torch.cat(parts).cpu().numpy()
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B.cpu().numpy(), nv)
    ok, bad = O.check_result(0, 0, A.nr, nv, ref, got)[:2]
    assert ok, f"{bad} elements off"
