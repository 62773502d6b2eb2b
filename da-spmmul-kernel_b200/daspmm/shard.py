"""Row sharding of one SpMM across ranks (one process per GPU).

The reference runs on one GPU.  The product C = A*B shards by output rows
with no exchange on the data path: rank r owns a contiguous row range of A
(rowPtr rebased to start at 0, the matching colIdx/values slice), B is
replicated -- broadcast once when a matrix becomes resident, not per call --
and each rank computes its rows of C with the single-GPU library.  If the
caller wants all of C on one rank, `gather_rows` collects the row blocks
there once (point-to-point sends, NCCL over NVLink on GPUs, gloo on CPUs).

For serving, the natural form is replicas: every rank runs its own server
over the matrices it owns (`owner_of`), and requests are routed by matrix id.

Ranges are balanced by nonzeros plus rows (each row costs one output row
store), split at row boundaries, deterministic in (rowPtr, world).
"""
from __future__ import annotations

import numpy as np

from . import Csr


def balanced_ranges(rowPtr: np.ndarray, parts: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [r0, r1) covering all rows, one per part, whose
    cost (nonzeros + rows) is as even as row boundaries allow: boundary k is
    the first row whose prefix cost reaches k/parts of the total."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    rp = np.asarray(rowPtr, dtype=np.int64)
    nr = rp.size - 1
    cost = rp + np.arange(nr + 1, dtype=np.int64)       # prefix cost at each row start
    total = int(cost[-1])
    cuts = [0]
    for k in range(1, parts):
        target = (total * k + parts - 1) // parts         # ceil(total * k / parts)
        cuts.append(int(np.searchsorted(cost, target, side="left")))
    cuts.append(nr)
    cuts = np.maximum.accumulate(np.minimum(np.array(cuts), nr))
    return [(int(cuts[i]), int(cuts[i + 1])) for i in range(parts)]


def shard(A: Csr, r0: int, r1: int) -> Csr:
    """Rows [r0, r1) of A as a standalone CSR (rowPtr rebased, same columns)."""
    k0, k1 = int(A.rowPtr[r0]), int(A.rowPtr[r1])
    rp = (A.rowPtr[r0: r1 + 1] - k0).astype(np.int32)
    return Csr(r1 - r0, A.nc, rp, A.colIdx[k0:k1].copy(), A.values[k0:k1].copy())


def owner_of(matrix_id: int, world: int) -> int:
    """Rank that keeps a pool matrix resident (replica-style serving)."""
    return int(matrix_id) % int(world)


def broadcast_dense(B, src: int = 0, group=None):
    """Replicates a dense operand once (torch.distributed broadcast; B must
    already have its final shape and dtype on every rank)."""
    import torch.distributed as dist
    dist.broadcast(B, src=src, group=group)
    return B


def gather_rows(C_local, row_counts: list[int], nv: int, dst: int = 0, group=None):
    """Concatenates every rank's C rows on rank `dst` (point-to-point; other
    ranks return None).  C_local: this rank's rows, flat row-major FP32."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if rank != dst:
        dist.send(C_local.contiguous(), dst=dst, group=group)
        return None
    parts = []
    for r in range(world):
        if r == rank:
            parts.append(C_local)
        else:
            buf = torch.empty(row_counts[r] * nv, dtype=C_local.dtype, device=C_local.device)
            dist.recv(buf, src=r, group=group)
            parts.append(buf)
    return torch.cat(parts)


class RowShardedSpmm:
    """One rank's part of C = A*B for a row-sharded A.

    `A` is the global host matrix (every rank builds or loads the same one);
    this rank keeps only its rows on `device`.  `spmm(B, C)` runs the
    library's balanced-CSR SpMM on this rank's rows (C holds rows
    [r0, r1) of the product)."""

    def __init__(self, A: Csr, rank: int, world: int, device="cuda"):
        from . import DeviceCsr
        self.ranges = balanced_ranges(A.rowPtr, world)
        self.r0, self.r1 = self.ranges[rank]
        self.local = shard(A, self.r0, self.r1)
        self.dev = DeviceCsr(self.local, device)
        self.row_counts = [b - a for a, b in self.ranges]

    def spmm(self, B, C, nv: int, beta: float = 0.0, stream=None):
        from . import Alg, spmm
        spmm(Alg.CSR_BALANCED, 0, self.dev, B, C, beta=beta, nv=nv, stream=stream)
