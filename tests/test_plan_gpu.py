"""Planned SpMM (daspmm_plan_*): the balanced split's boundaries computed once,
each product one launch of the window kernel.  Against the stateless
daspmm_spmm with the same configuration the products are bit-identical (same
chunks, same order of summation), call after call -- which also shows that the
window kernel leaves its queue heads and split-row counters at zero -- and
across the calls a plan hands to the stateless path (beta != 0, misaligned
C).  The first product of each case is also checked against the oracle."""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mats():
    rng = np.random.default_rng(17)
    lens = rng.integers(0, 4, 400)
    lens[:3] = 0
    lens[50] = 3000           # a hub row split across many chunks
    lens[-5:] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(4000, int(k), replace=False)) for k in lens]
                        ).astype(np.int32)
    va = rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)
    return {"powerlaw": D.gen_powerlaw(20000, dmax=2000, seed=8),
            "random_empty_rows": D.gen_random(5000, 4000, 3.0, seed=9),
            "hub": D.Csr(400, 4000, rp, ci, va)}


def _check(A, nv, B, C, beta=0.0, C0=None, what=""):
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    c64, absc = O.spmm_f64(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    if beta != 0.0:
        ref = ref + np.float32(beta) * C0
        c64 = c64 + beta * C0.astype(np.float64)
        absc = absc + abs(beta) * np.abs(C0.astype(np.float64))
    ok, bad = O.check_result(0, 0, A.nr, nv, ref, C, O.REF_ABS_TOL)
    assert ok, f"{what}: differs from the oracle at {bad}"
    assert O.rel_err(C, c64, absc) <= O.REL_TOL_F32, what


@pytest.mark.parametrize("name", ["powerlaw", "random_empty_rows", "hub"])
def test_plan_equals_stateless(cuda, name):
    import torch
    A = _mats()[name]
    dA = D.DeviceCsr(A)
    rng = np.random.default_rng(5)
    for nv in (32, 64, 128, 256):
        plan = D.Plan(dA, nv)
        cfg = plan.config()
        Cs = torch.empty(A.nr * nv, device="cuda")
        Cp = torch.empty(A.nr * nv, device="cuda")
        for it in range(3):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            Bt = torch.from_numpy(B).cuda()
            Cp.fill_(float("nan"))
            plan.spmm(Bt, Cp)
            D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, Cs, nv=nv, cfg=cfg)
            torch.cuda.synchronize()
            assert torch.equal(Cp, Cs), f"{name} nv={nv} call {it}"
            if it == 0:
                _check(A, nv, B, Cp.cpu().numpy(), what=f"{name} nv={nv}")
        # beta != 0 (the stateless path on the plan's workspace), then beta = 0 again
        C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
        Cp.copy_(torch.from_numpy(C0))
        Cs.copy_(torch.from_numpy(C0))
        plan.spmm(Bt, Cp, beta=0.5)
        D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, Cs, beta=0.5, nv=nv, cfg=cfg)
        torch.cuda.synchronize()
        assert torch.equal(Cp, Cs), f"{name} nv={nv} beta"
        _check(A, nv, B, Cp.cpu().numpy(), beta=0.5, C0=C0, what=f"{name} nv={nv} beta")
        # C 16 bytes off 32-byte alignment: the stateless path
        Cbuf = torch.full((A.nr * nv + 8,), float("nan"), device="cuda")
        Co = Cbuf[4:4 + A.nr * nv]
        plan.spmm(Bt, Co)
        plan.spmm(Bt, Cp)
        D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, Cs, nv=nv, cfg=cfg)
        torch.cuda.synchronize()
        assert torch.equal(Co, Cs) and torch.equal(Cp, Cs), f"{name} nv={nv} after fallback"
        plan.close()


def test_plan_full_size_power_law(cuda):
    """The 262,144-row power-law matrix at N = 128: ten planned products in a
    row, each bit-identical to the stateless call."""
    import torch
    A = D.gen_powerlaw(262144, seed=0)
    dA = D.DeviceCsr(A)
    nv = 128
    plan = D.Plan(dA, nv)
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    Cs = torch.empty(A.nr * nv, device="cuda")
    Cp = torch.empty(A.nr * nv, device="cuda")
    for it in range(10):
        Bt = torch.empty(A.nc * nv, device="cuda").uniform_(-1, 1, generator=g)
        plan.spmm(Bt, Cp)
        D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, Cs, nv=nv)
        torch.cuda.synchronize()
        assert torch.equal(Cp, Cs), f"call {it}"
    B = Bt.cpu().numpy()
    ok, bad = O.check_result(0, 0, A.nr, nv,
                             O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv),
                             Cp.cpu().numpy(), O.REF_ABS_TOL)
    assert ok, bad
    plan.close()


def test_plan_rejects_other_algorithms(cuda):
    A = D.gen_uniform(100, 100, 4, seed=1)
    dA = D.DeviceCsr(A)
    with pytest.raises(D.DaspmmError):
        D.Plan(dA, 32, cfg=D.Config(alg=int(D.Alg.CSR_SCALAR)))


def test_plan_non_finite_row0(cuda):
    """Row 0 of B holds Inf / NaN and no nonzero references it: the window
    kernel pads with column 0, so every chunk goes to the walk (in plan mode
    the walk kernel sees row 0 itself); the product stays finite and equal to
    the stateless call's, and the next finite B runs the window kernel again."""
    import torch
    base = D.gen_powerlaw(6000, dmax=600, seed=12)
    A = D.Csr(base.nr, base.nc + 1, base.rowPtr, base.colIdx + 1, base.values)
    dA = D.DeviceCsr(A)
    rng = np.random.default_rng(2)
    nv = 128
    plan = D.Plan(dA, nv)
    cfg = plan.config()
    for bad in (float("inf"), float("nan"), None):
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        if bad is not None:
            B[:nv] = bad
        Bt = torch.from_numpy(B).cuda()
        Cp = torch.full((A.nr * nv,), float("nan"), device="cuda")
        Cs = torch.full((A.nr * nv,), float("nan"), device="cuda")
        plan.spmm(Bt, Cp)
        D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, Cs, nv=nv, cfg=cfg)
        torch.cuda.synchronize()
        assert torch.equal(Cp, Cs), f"row 0 = {bad}"
        assert bool(torch.isfinite(Cp).all())
        _check(A, nv, B, Cp.cpu().numpy(), what=f"plan row 0 = {bad}")
    plan.close()
