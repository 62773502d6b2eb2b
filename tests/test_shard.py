"""Row sharding across ranks (CPU: gloo, world size 2 and 3).

The multi-GPU form of the path has no exchange on the data path: ranks own
contiguous row ranges, B is broadcast once, and C may be gathered once.  These
tests run that host logic with the gloo backend; each rank computes its rows
with the oracle (CPU), and rank 0 checks the gathered product against the
oracle's product of the whole matrix, bit for bit (rows are independent).
"""
import os
import socket

import numpy as np
import pytest

import daspmm as D
from daspmm import shard as S


def _matrix():
    return D.gen_powerlaw(3000, dmax=400, seed=9)


def test_balanced_ranges_cover_and_balance():
    A = _matrix()
    lens = np.diff(A.rowPtr)
    total = A.nnz + A.nr
    for parts in (1, 2, 3, 7, 64):
        rg = S.balanced_ranges(A.rowPtr, parts)
        assert len(rg) == parts and rg[0][0] == 0 and rg[-1][1] == A.nr
        assert all(rg[i][1] == rg[i + 1][0] for i in range(parts - 1))
        for a, b in rg:
            assert a <= b
            cost = int(A.rowPtr[b] - A.rowPtr[a]) + (b - a)
            assert cost <= total / parts + lens.max() + 1
    assert S.balanced_ranges(A.rowPtr, 4) == S.balanced_ranges(A.rowPtr.copy(), 4)
    # more parts than rows: empty ranges, still a cover
    tiny = D.Csr(2, 5, np.array([0, 1, 3], np.int32), np.array([0, 1, 4], np.int32),
                 np.ones(3, np.float32))
    rg = S.balanced_ranges(tiny.rowPtr, 5)
    assert rg[0][0] == 0 and rg[-1][1] == 2 and sum(b - a for a, b in rg) == 2


def test_shards_reassemble():
    A = _matrix()
    rg = S.balanced_ranges(A.rowPtr, 3)
    parts = [S.shard(A, a, b) for a, b in rg]
    for p in parts:
        assert p.rowPtr[0] == 0 and p.rowPtr[-1] == p.colIdx.size == p.values.size
    rp = np.concatenate([[0]] + [p.rowPtr[1:] + off for p, off in
                                 zip(parts, np.cumsum([0] + [p.nnz for p in parts[:-1]]))])
    assert np.array_equal(rp, A.rowPtr)
    assert np.array_equal(np.concatenate([p.colIdx for p in parts]), A.colIdx)
    assert np.array_equal(np.concatenate([p.values for p in parts]), A.values)


def test_owner_routing():
    world = 4
    owners = [S.owner_of(m, world) for m in range(64)]
    assert all(0 <= o < world for o in owners)
    assert [owners.count(r) for r in range(world)] == [16] * world


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nv):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = _matrix()
        rg = S.balanced_ranges(A.rowPtr, world)
        r0, r1 = rg[rank]
        local = S.shard(A, r0, r1)
        B = torch.zeros(A.nc * nv, dtype=torch.float32)
        if rank == 0:
            B.copy_(torch.from_numpy(D.gen_dense(A.nc * nv, seed=3)))
        S.broadcast_dense(B, src=0)                      # B replicated once
        C = O.spmm_f32(0, local.nr, local.nc, local.rowPtr, local.colIdx, local.values,
                       B.numpy(), nv)
        full = S.gather_rows(torch.from_numpy(C), [b - a for a, b in rg], nv, dst=0)
        if rank == 0:
            ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B.numpy(), nv)
            assert full.numel() == A.nr * nv
            assert np.array_equal(full.numpy(), ref), "gathered shards differ from the product"
        # replica routing: every request is answered once, by its owner
        reqs = list(range(24))
        mine = [m for m in reqs if S.owner_of(m, world) == rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        assert sorted(sum(got, [])) == reqs
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_row_shards_match_oracle(world):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), 32), nprocs=world, join=True)
