"""Serving loop (daspmm_server_*) on the GPU.

Every served result is checked against the oracle (FP32 storage: the
reference's 1e-3 rule; BF16 B: 2e-5 relative to sum|a||b| against FP64 of
the dequantized inputs), results are bit-identical whether a request runs
alone or inside a Poisson-arriving mix, and the admission / cancellation /
validation paths fail the way the header says: over-budget requests are
refused before any device work, a queued request waits for budget and can
be cancelled, malformed matrices are rejected when added.
"""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pool(rng, n=8):
    mats = []
    for i in range(n):
        if i % 3 == 0:
            mats.append(D.gen_powerlaw(int(rng.integers(500, 6000)), dmax=int(rng.integers(50, 900)),
                                       seed=40 + i))
        elif i % 3 == 1:
            r = int(rng.integers(300, 5000))
            mats.append(D.gen_random(r, r, float(rng.uniform(1, 12)), seed=40 + i))
        else:
            r = int(rng.integers(64, 3000))
            mats.append(D.gen_uniform(r, r, int(rng.integers(1, 30)), seed=40 + i))
    return mats


def _b_for(A, nv, b_fmt, rng):
    import torch
    B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
    Bt = torch.from_numpy(B).cuda()
    if b_fmt == D.Fmt.F32:
        return Bt, B.astype(np.float64)
    q = D.quantize(Bt, D.Fmt.BF16)
    return q, O.dequantize(1, q.cpu().view(torch.int16).numpy().view(np.uint16))


def _check(A, nv, got, b64, b_fmt):
    c64, absc = O.spmm_f64d(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values.astype(np.float64),
                            b64, nv)
    e = O.rel_err(got, c64, absc)
    assert e <= O.REL_TOL_F32, f"nr={A.nr} nnz={A.nnz} nv={nv}: rel err {e}"
    if b_fmt == D.Fmt.F32:
        ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, b64.astype(np.float32), nv)
        assert O.check_result(0, 0, A.nr, nv, ref, got)[0]


def _setup(mode, b_fmt, rng, budget=1 << 28, **kw):
    mats = _pool(rng)
    srv = D.Server(budget_bytes=budget, mode=mode, b_fmt=b_fmt, **kw)
    dev = [D.DeviceCsr(A) for A in mats]
    ids = [srv.add_matrix(dA) for dA in dev]
    return srv, mats, dev, ids


@pytest.mark.parametrize("mode,b_fmt", [(D.ServeMode.BATCHED, D.Fmt.F32),
                                        (D.ServeMode.BATCHED, D.Fmt.BF16),
                                        (D.ServeMode.PLAIN, D.Fmt.F32)])
def test_served_results_match_oracle(cuda, mode, b_fmt):
    import torch
    rng = np.random.default_rng(11)
    srv, mats, dev, ids = _setup(mode, b_fmt, rng)
    reqs = []
    for k in range(30):
        m = int(rng.integers(0, len(mats)))
        nv = int(rng.choice([16, 64, 256, 32, 96]))
        B, b64 = _b_for(mats[m], nv, b_fmt, rng)
        reqs.append((m, nv, B, b64))
    tickets = [srv.submit(ids[m], nv, B) for m, nv, B, _ in reqs]
    for t, (m, nv, B, b64) in zip(tickets, reqs):
        st, res = srv.wait(t, 20000)
        assert st == 0 and res.status == 0
        C = srv.result_tensor(res, mats[m].nr, nv)
        torch.cuda.synchronize()
        _check(mats[m], nv, C.cpu().numpy(), b64, b_fmt)
        srv.release(t)
    s = srv.stats()
    assert s["completed"] == 30 and s["arena_used"] == 0 and s["error"] == 0
    srv.close()


def test_alone_equals_in_the_mix(cuda):
    import torch
    rng = np.random.default_rng(5)
    srv, mats, dev, ids = _setup(D.ServeMode.BATCHED, D.Fmt.BF16, rng, budget=1 << 30)
    reqs = []
    for k in range(40):
        m = int(rng.integers(0, len(mats)))
        nv = int(rng.choice([16, 64, 256]))
        B, _ = _b_for(mats[m], nv, D.Fmt.BF16, rng)
        reqs.append((ids[m], nv, B))
    alone = []
    for m, nv, B in reqs:                      # one at a time: groups of one
        t = srv.submit(m, nv, B)
        st, res = srv.wait(t, 20000)
        assert st == 0 and res.status == 0
        alone.append(srv.result_tensor(res, mats[m].nr, nv).clone())
        srv.release(t)
    arrivals = np.cumsum(rng.exponential(1.0 / 2e6, len(reqs)))   # dense: groups form
    res = srv.replay(reqs, arrivals, release=False)
    groups = {r.group for r in res}
    assert len(groups) < len(reqs), "the mix never batched two requests"
    for (m, nv, B), r, a in zip(reqs, res, alone):
        assert r.status == 0
        got = srv.result_tensor(r, mats[m].nr, nv)
        assert torch.equal(got, a), "result differs alone vs in the mix"
    st = srv.stats()
    assert st["arena_used"] > 0
    srv.close()


def test_admission_budget_and_cancel(cuda):
    import torch
    rng = np.random.default_rng(2)
    A = D.gen_uniform(4096, 4096, 8, seed=3)
    dA = D.DeviceCsr(A)
    nv = 64
    cbytes = A.nr * nv * 4                     # 1 MiB
    srv = D.Server(budget_bytes=int(cbytes * 1.5), mode=D.ServeMode.BATCHED)
    m = srv.add_matrix(dA)
    B = torch.from_numpy(rng.uniform(-1, 1, A.nc * nv).astype(np.float32)).cuda()
    with pytest.raises(D.DaspmmError) as ei:   # C alone exceeds the budget
        srv.submit(m, 128, torch.zeros(A.nc * 128, device="cuda"))
    assert ei.value.status == 7
    t1 = srv.submit(m, nv, B)
    st, r1 = srv.wait(t1, 20000)
    assert st == 0 and r1.status == 0
    t2 = srv.submit(m, nv, B)                  # does not fit while t1's C is held
    st, r2 = srv.wait(t2, 200)
    assert st == 6 and r2.status == -1         # DASPMM_ERR_TIMEOUT, still queued
    assert srv.stats()["queued"] == 1
    t3 = srv.submit(m, nv, B)
    assert srv.cancel(t3) == 0                 # queued behind t2: cancellable
    st, r3 = srv.wait(t3, 1000)
    assert st == 0 and r3.status == 8          # DASPMM_ERR_CANCELLED
    c1 = srv.result_tensor(r1, A.nr, nv).clone()
    srv.release(t1)                            # frees budget: t2 runs
    st, r2 = srv.wait(t2, 20000)
    assert st == 0 and r2.status == 0
    assert srv.cancel(t2) == 2                 # finished: not cancellable
    assert torch.equal(srv.result_tensor(r2, A.nr, nv), c1)
    srv.release(t2)
    srv.release(t3)
    s = srv.stats()
    assert s["refused"] == 1 and s["cancelled"] == 1 and s["arena_used"] == 0
    srv.close()


def test_destroy_cancels_queued(cuda):
    import torch
    A = D.gen_uniform(2048, 2048, 4, seed=1)
    dA = D.DeviceCsr(A)
    srv = D.Server(budget_bytes=A.nr * 32 * 4, mode=D.ServeMode.PLAIN)
    m = srv.add_matrix(dA)
    B = torch.ones(A.nc * 32, device="cuda")
    t1 = srv.submit(m, 32, B)
    st, r1 = srv.wait(t1, 20000)
    assert r1.status == 0
    srv.submit(m, 32, B)                       # waits for budget forever
    srv.close()                                # returns: the queued request is cancelled


def _raw(nr, nc, rowPtr, colIdx, nnz):
    """A device CSR whose nnz is given, not taken from rowPtr (for malformed cases)."""
    import torch
    from types import SimpleNamespace
    return SimpleNamespace(nr=nr, nc=nc, nnz=nnz, rowPtr=torch.from_numpy(rowPtr).cuda(),
                           colIdx=torch.from_numpy(colIdx).cuda(),
                           values=torch.ones(max(1, nnz), device="cuda"))


def test_malformed_matrices_rejected(cuda):
    import torch
    srv = D.Server(budget_bytes=1 << 20)
    good = D.gen_uniform(100, 50, 3, seed=2)
    nnz = good.nnz
    assert D.csr_check(_raw(100, 50, good.rowPtr, good.colIdx, nnz), sorted_cols=True) == -1
    ci = good.colIdx.copy()
    ci[40] = 50                                # out of range, row 13
    bad_col = _raw(100, 50, good.rowPtr, ci, nnz)
    assert D.csr_check(bad_col) == 13
    with pytest.raises(D.DaspmmError) as ei:
        srv.add_matrix(bad_col)
    assert ei.value.status == 9
    ci = good.colIdx.copy()
    ci[41] = -1
    assert D.csr_check(_raw(100, 50, good.rowPtr, ci, nnz)) == 13
    rp = good.rowPtr.copy()
    rp[30] = rp[31] + 1                        # decreasing at row 30
    assert D.csr_check(_raw(100, 50, rp, good.colIdx, nnz)) == 30
    rp = good.rowPtr.copy()
    rp[0] = 1                                  # rowPtr[0] != 0
    assert D.csr_check(_raw(100, 50, rp, good.colIdx, nnz)) == 0
    rp = good.rowPtr.copy()
    rp[-1] -= 1                                # rowPtr[nr] != nnz
    assert D.csr_check(_raw(100, 50, rp, good.colIdx, nnz)) == 99
    ci = good.colIdx.copy()
    a = int(good.rowPtr[7])
    ci[a], ci[a + 1] = ci[a + 1], ci[a]        # unsorted inside row 7
    un = _raw(100, 50, good.rowPtr, ci, nnz)
    assert D.csr_check(un) == -1 and D.csr_check(un, sorted_cols=True) == 7
    assert srv.add_matrix(un) == 0             # the server needs ranges, not order
    with pytest.raises(D.DaspmmError):
        srv.submit(5, 32, torch.zeros(1, device="cuda"))   # unknown matrix id
    srv.close()
