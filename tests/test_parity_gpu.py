"""GPU parity: every algorithm x layout x nv through the C ABI against the
oracle (the reference's host loop restated, pinned in test_oracle.py).

Tolerances (stated once, in oracle/oracle.py):
  * reference rule  |gpu - host_fp32| <= 1e-3   (checkResult, spmvspmm_benchmark.cu:94)
  * FP64 rule       |gpu - c64| <= 2e-5 * sum_p |a_p||b_p|
Index and partition arithmetic is compared bit for bit.
"""
import os

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALGS = [D.Alg.CSR_SCALAR, D.Alg.CSR_VECTOR, D.Alg.COO_SCALAR, D.Alg.COO_VECTOR,
        D.Alg.CSR_BALANCED]
NVS = [1, 2, 3, 4, 8, 16, 32, 64, 128]


def _dev(A):
    return D.DeviceCsr(A)


def _run(A, dA, alg, layout, nv, B, beta=0.0, C0=None, cfg=None):
    import torch
    Bt = torch.from_numpy(np.ascontiguousarray(B, np.float32)).cuda()
    if C0 is None:
        Ct = torch.full((A.nr * nv,), float("nan"), dtype=torch.float32, device="cuda")
        if beta != 0.0:
            Ct.zero_()
    else:
        Ct = torch.from_numpy(np.ascontiguousarray(C0, np.float32)).cuda()
    if cfg is not None:
        cfg.alg = int(alg)
    D.spmm(alg, layout, dA, Bt, Ct, beta=beta, nv=nv, cfg=cfg)
    torch.cuda.synchronize()
    return Ct.cpu().numpy()


def _check(A, layout, nv, B, C, beta=0.0, C0=None, what=""):
    ref = O.spmm_f32(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    c64, absc = O.spmm_f64(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    if beta != 0.0:
        ref = ref + np.float32(beta) * C0
        c64 = c64 + beta * C0.astype(np.float64)
        absc = absc + abs(beta) * np.abs(C0.astype(np.float64))
    ok, bad = O.check_result(layout, layout, A.nr, nv, ref, C, O.REF_ABS_TOL)
    assert ok, f"{what}: reference 1e-3 rule fails at {bad}"
    e = O.rel_err(C, c64, absc)
    assert e <= O.REL_TOL_F32, f"{what}: rel err {e}"


@pytest.fixture(scope="module")
def mats(cuda):
    rng = np.random.default_rng(4)
    out = {
        "uniform": D.gen_uniform(300, 257, 16, seed=0),
        "powerlaw": D.gen_powerlaw(3000, dmax=700, seed=1),
        "random": D.gen_random(500, 400, 3.0, seed=2),   # includes empty rows
    }
    # a matrix with one hub row longer than several chunks and empty tails
    lens = rng.integers(0, 4, 257)
    lens[:5] = 0
    lens[100] = 1500
    lens[-7:] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(2000, int(k), replace=False)) for k in lens]
                        ).astype(np.int32)
    va = rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)
    out["hub"] = D.Csr(257, 2000, rp, ci, va)
    return {k: (A, _dev(A)) for k, A in out.items()}


@pytest.mark.parametrize("name", ["uniform", "powerlaw", "random", "hub"])
@pytest.mark.parametrize("layout", [0, 1])
def test_all_algs_all_nv(mats, name, layout):
    A, dA = mats[name]
    rng = np.random.default_rng(11)
    for nv in NVS:
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        for alg in ALGS:
            C = _run(A, dA, alg, layout, nv, B)
            _check(A, layout, nv, B, C, what=f"{name} alg={alg.name} layout={layout} nv={nv}")


def test_golden_reference_outputs(cuda, golden_dir):
    """GPU results against the reference's own host outputs (committed)."""
    g = np.load(os.path.join(golden_dir, "golden_spmm.npz"))
    for name in ("uniform", "powerlaw", "ragged"):
        nr, nc = (int(x) for x in g[f"{name}_dims"])
        A = D.Csr(nr, nc, g[f"{name}_rowPtr"], g[f"{name}_colIdx"], g[f"{name}_values"])
        dA = _dev(A)
        for f in g.files:
            if not f.startswith(f"{name}_C_"):
                continue
            _, _, tag, nv = f.split("_")
            nv, lay = int(nv), (0 if tag == "rm" else 1)
            B = g[f"{name}_B"][: nc * nv]
            for alg in ALGS:
                C = _run(A, dA, alg, lay, nv, B)
                ok, bad = O.check_result(lay, lay, nr, nv, g[f], C, 1e-3)
                assert ok, f"{f} alg={alg.name} at {bad}"


def test_compat_semantics(mats):
    """cudaSpmm<256,32>: CSR overwrites C, COO adds into C (spmvspmm.h:53-199)."""
    import torch
    A, dA = mats["powerlaw"]
    rng = np.random.default_rng(3)
    for layout in (0, 1):
        for nv in (1, 4, 32):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
            ref = O.spmm_f32(layout, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
            Bt = torch.from_numpy(B).cuda()
            for alg in (0, 1, 2, 3):
                Ct = torch.from_numpy(C0).cuda()
                assert D.compat_spmm(alg, layout, dA, Bt, Ct, nv) == 0
                torch.cuda.synchronize()
                want = ref if alg < 2 else ref + C0
                ok, bad = O.check_result(layout, layout, A.nr, nv, want, Ct.cpu().numpy())
                assert ok, (layout, nv, alg, bad)


@pytest.mark.parametrize("beta", [1.0, -0.5, 2.0])
def test_beta(mats, beta):
    A, dA = mats["hub"]
    rng = np.random.default_rng(5)
    for layout in (0, 1):
        nv = 8
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
        for alg in ALGS:
            C = _run(A, dA, alg, layout, nv, B, beta=beta, C0=C0)
            _check(A, layout, nv, B, C, beta=beta, C0=C0, what=f"beta={beta} alg={alg.name}")


def test_design_space_points(mats):
    """Explicit (vec, L, S, CF, chunk, snap, block) points all give the product."""
    A, dA = mats["powerlaw"]
    rng = np.random.default_rng(6)
    nv = 64
    B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
    pts = []
    for vec in (1, 2, 4):
        for cf in (1, 2):
            for L in (1, 4, 8, 32):
                pts.append((D.Alg.CSR_SCALAR, dict(vec=vec, cf=cf, lanes_col=L, lanes_nnz=1)))
                pts.append((D.Alg.COO_SCALAR, dict(vec=vec, cf=cf, lanes_col=L, chunk=17)))
                pts.append((D.Alg.CSR_BALANCED, dict(vec=vec, cf=cf, lanes_col=L, chunk=40,
                                                     snap=9)))
                S = 32 // L
                if S > 1:
                    pts.append((D.Alg.CSR_VECTOR, dict(vec=vec, cf=cf, lanes_col=L, lanes_nnz=S)))
                    pts.append((D.Alg.COO_VECTOR, dict(vec=vec, cf=cf, lanes_col=L, lanes_nnz=S,
                                                       chunk=4 * S)))
    pts.append((D.Alg.CSR_BALANCED, dict(chunk=1, snap=1)))
    pts.append((D.Alg.CSR_BALANCED, dict(chunk=4096, snap=4096, block=128)))
    pts.append((D.Alg.COO_SCALAR, dict(chunk=1, block=128)))
    for alg, kw in pts:
        cfg = D.Config(alg=int(alg), **kw)
        C = _run(A, dA, alg, 0, nv, B, cfg=cfg)
        _check(A, 0, nv, B, C, what=f"{alg.name} {kw}")
    for cf in (1, 2, 4, 8):   # col-major coarsening
        for alg, extra in ((D.Alg.CSR_SCALAR, {}), (D.Alg.CSR_VECTOR, dict(lanes_nnz=8)),
                           (D.Alg.COO_SCALAR, dict(chunk=9)),
                           (D.Alg.COO_VECTOR, dict(lanes_nnz=16, chunk=32)),
                           (D.Alg.CSR_BALANCED, dict(chunk=33, snap=5))):
            cfg = D.Config(alg=int(alg), cf=cf, **extra)
            C = _run(A, dA, alg, 1, nv, B, cfg=cfg)
            _check(A, 1, nv, B, C, what=f"CM {alg.name} cf={cf}")


@pytest.mark.parametrize("name", ["powerlaw", "hub", "uniform", "random"])
def test_balanced_tma_ring(mats, name):
    """The TMA-fed ring (pipe 2) against the oracle: tile widths 32/64/128,
    several column tiles, chunk sizes that split hub rows across many chunks,
    beta, and no expired device waits."""
    A, dA = mats[name]
    rng = np.random.default_rng(12)
    for pipe in (2, 3, 4):   # TMA ring / cp.async ring / lean register gather
        for nv in (32, 64, 96, 128, 160, 192, 256):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            for kw in ({}, dict(chunk=40, snap=9), dict(chunk=7, snap=3), dict(chunk=5000),
                       dict(lanes_col=8, chunk=50)):   # 32-float tiles
                cfg = D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=pipe, **kw)
                C = _run(A, dA, D.Alg.CSR_BALANCED, 0, nv, B, cfg=cfg)
                _check(A, 0, nv, B, C, what=f"ring{pipe} {name} nv={nv} {kw}")
        nv = 64
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
        cfg = D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=pipe, chunk=33, snap=5)
        C = _run(A, dA, D.Alg.CSR_BALANCED, 0, nv, B, beta=0.75, C0=C0, cfg=cfg)
        _check(A, 0, nv, B, C, beta=0.75, C0=C0, what=f"ring{pipe} beta")
    assert D.lib().daspmm_device_error() == 0


def test_deterministic_repeat(mats):
    A, dA = mats["hub"]
    B = np.random.default_rng(8).uniform(-1, 1, A.nc * 32).astype(np.float32)
    for alg in ALGS:
        c1 = _run(A, dA, alg, 0, 32, B)
        c2 = _run(A, dA, alg, 0, 32, B)
        np.testing.assert_array_equal(c1, c2)
    for pipe in (1, 2, 4):
        cfg = lambda: D.Config(alg=int(D.Alg.CSR_BALANCED), pipe=pipe, chunk=64)
        c1 = _run(A, dA, D.Alg.CSR_BALANCED, 0, 32, B, cfg=cfg())
        c2 = _run(A, dA, D.Alg.CSR_BALANCED, 0, 32, B, cfg=cfg())
        np.testing.assert_array_equal(c1, c2)


def test_edge_cases(cuda):
    rng = np.random.default_rng(9)
    cases = []
    cases.append(D.Csr(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                       np.array([2.5], np.float32)))
    cases.append(D.Csr(5, 3, np.zeros(6, np.int32), np.zeros(0, np.int32),
                       np.zeros(0, np.float32)))                     # nnz == 0
    cases.append(D.Csr(4, 1, np.array([0, 1, 2, 3, 4], np.int32), np.zeros(4, np.int32),
                       np.ones(4, np.float32)))                      # single column
    n = 4096                                                         # one full row
    cases.append(D.Csr(3, n, np.array([0, 0, n, n], np.int32), np.arange(n, dtype=np.int32),
                       rng.uniform(-1, 1, n).astype(np.float32)))
    for A in cases:
        dA = _dev(A)
        for nv in (1, 5, 32, 128):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            for layout in (0, 1):
                for alg in ALGS:
                    C = _run(A, dA, alg, layout, nv, B)
                    _check(A, layout, nv, B, C, what=f"edge nr={A.nr} nnz={A.nnz} {alg.name}")


def test_no_columns_no_nonzeros(cuda):
    """nr > 0 rows, no nonzeros and no columns: B has no rows, so nothing may
    be read from it (the caller's pointer is valid but holds no row); C = 0
    (beta = 0) or beta * C."""
    import torch
    A = D.Csr(6, 0, np.zeros(7, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    dA = _dev(A)
    Bt = torch.zeros(1, device="cuda")   # a valid pointer to no B row
    for nv in (1, 32, 128):
        for layout in (0, 1):
            for alg in ALGS:
                for beta in (0.0, 0.5):
                    C = torch.full((A.nr * nv,), 2.0, device="cuda")
                    D.spmm(alg, layout, dA, Bt, C, beta=beta, nv=nv)
                    torch.cuda.synchronize()
                    assert torch.all(C == 2.0 * beta), f"{alg.name} layout {layout} nv {nv}"


def test_l2_window_knob(cuda):
    """An L2 access-policy window over B (config l2_window, with a persisting
    set-aside) changes where B's lines live in L2, not the arithmetic: the
    products are bit-identical with and without it, FP32 and BF16 storage."""
    import torch
    L = D.lib()
    A = D.gen_powerlaw(20000, dmax=2000, seed=8)
    dA = D.DeviceCsr(A)
    rng = np.random.default_rng(8)
    try:
        assert L.daspmm_l2_set_aside(32 << 20) == 0
        for nv in (64, 128, 256):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            Bt = torch.from_numpy(B).cuda()
            ref = torch.empty(A.nr * nv, device="cuda")
            D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, ref, nv=nv, cfg=D.Config(alg=4))
            b16 = D.quantize(Bt, D.Fmt.BF16)
            v16 = D.quantize(dA.values, D.Fmt.BF16)
            ref16 = torch.empty(A.nr * nv, device="cuda")
            D.spmm_mixed(dA, v16, D.Fmt.BF16, b16, D.Fmt.BF16, ref16, nv)
            for w in (250, 1000):
                C = torch.full((A.nr * nv,), float("nan"), device="cuda")
                D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, C, nv=nv, cfg=D.Config(alg=4, l2_window=w))
                C16 = torch.full((A.nr * nv,), float("nan"), device="cuda")
                D.spmm_mixed(dA, v16, D.Fmt.BF16, b16, D.Fmt.BF16, C16, nv,
                             cfg=D.Config(alg=4, l2_window=w))
                torch.cuda.synchronize()
                assert torch.equal(C, ref), f"nv={nv} window {w}"
                assert torch.equal(C16, ref16), f"BF16 nv={nv} window {w}"
            _check(A, 0, nv, B, ref.cpu().numpy(), what=f"l2 window nv={nv}")
        bad = torch.empty(A.nr * 64, device="cuda")
        with pytest.raises(D.DaspmmError):
            D.spmm(D.Alg.CSR_BALANCED, 0, dA, Bt, bad, nv=64, cfg=D.Config(alg=4, l2_window=1001))
    finally:
        assert L.daspmm_l2_set_aside(0) == 0


def test_partition_bit_exact(mats):
    for name in ("uniform", "powerlaw", "random", "hub"):
        A, dA = mats[name]
        for chunk, snap in ((128, 64), (32, 16), (7, 7), (1, 1), (1000, 300)):
            got = D.partition(dA, chunk, snap).cpu().numpy()
            want = O.balanced_partition(A.nr, A.rowPtr, chunk, snap)
            np.testing.assert_array_equal(got, want, err_msg=f"{name} {chunk} {snap}")


def test_ownership_bit_exact(mats):
    for name in ("uniform", "powerlaw", "random", "hub"):
        A, dA = mats[name]
        for chunk, snap in ((128, 64), (32, 16), (5, 2), (1, 1)):
            got = D.ownership(D.Alg.CSR_BALANCED, dA, chunk, snap).cpu().numpy()
            want = O.balanced_ownership(A.nr, A.rowPtr, chunk, snap)
            np.testing.assert_array_equal(got, want, err_msg=f"bal {name} {chunk}")
            got = D.ownership(D.Alg.COO_SCALAR, dA, chunk).cpu().numpy()
            want = O.coo_ownership(A.nr, A.rowIdx, chunk)
            np.testing.assert_array_equal(got, want, err_msg=f"coo {name} {chunk}")


def test_coo_to_csr_bit_exact(cuda, golden_dir):
    import torch
    g = np.load(os.path.join(golden_dir, "golden_rowptr.npz"))
    i = 0
    while f"nr_{i}" in g.files:
        nr = int(g[f"nr_{i}"][0])
        ri = torch.from_numpy(g[f"rowIdx_{i}"]).cuda()
        np.testing.assert_array_equal(D.coo_to_csr(nr, ri).cpu().numpy(), g[f"rowPtr_{i}"])
        i += 1
    A = D.gen_powerlaw(50000, seed=3)
    got = D.coo_to_csr(A.nr, torch.from_numpy(A.rowIdx).cuda()).cpu().numpy()
    np.testing.assert_array_equal(got, A.rowPtr)
    empty = torch.zeros(0, dtype=torch.int32, device="cuda")
    np.testing.assert_array_equal(D.coo_to_csr(6, empty).cpu().numpy(), np.zeros(7, np.int32))


@pytest.mark.slow
def test_full_size_configs(cuda):
    """The benchmark shapes at full size against the oracle."""
    A1 = D.gen_uniform(4096, 4096, 16, seed=0)
    d1 = _dev(A1)
    for nv in (1, 32):
        B = D.gen_dense(A1.nc * nv, seed=1)
        for alg in ALGS:
            C = _run(A1, d1, alg, 0, nv, B)
            _check(A1, 0, nv, B, C, what=f"cfg1 nv={nv} {alg.name}")
    A2 = D.gen_powerlaw(262144, seed=0)
    d2 = _dev(A2)
    nv = 128
    B = D.gen_dense(A2.nc * nv, seed=1)
    for alg in (D.Alg.CSR_BALANCED, D.Alg.CSR_SCALAR, D.Alg.COO_SCALAR):
        C = _run(A2, d2, alg, 0, nv, B)
        _check(A2, 0, nv, B, C, what=f"cfg2 {alg.name}")


def _sparse_empty_rows(nr, nc, seed):
    """Rows of 1-3 nonzeros with about 1 % empty rows and a few hub rows: a
    chunk's empty row often lies far beyond its first rows, so the window
    kernels' scan for it runs several steps."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(1, 4, nr)
    lens[rng.random(nr) < 0.01] = 0
    lens[rng.integers(0, nr, 4)] = 700
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(nc, int(k), replace=False)) for k in lens]
                        ).astype(np.int32)
    va = rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)
    return D.Csr(nr, nc, rp, ci, va)


def test_group_kernel_equals_32_lane_kernel(cuda):
    """FP32 row-major balanced CSR: with B and C 32-byte aligned the worker-
    group window kernel runs (G = 16 / 8 / 8 lanes per chunk for 128 / 64 /
    32-column tiles), with both 16 bytes off that alignment the 32-lane one.
    Same chunks and order of summation: the products are bit-identical,
    whatever the tile width.  The third matrix puts empty rows deep inside
    chunks: both kernels must hand exactly those chunks to the walk kernel."""
    import torch
    rng = np.random.default_rng(12)
    for A in (D.gen_powerlaw(20000, dmax=2000, seed=8), D.gen_random(5000, 4000, 5.0, seed=9),
              _sparse_empty_rows(6000, 5000, 13)):
        dA = D.DeviceCsr(A)
        for nv in (32, 64, 96, 128, 256):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            Ba = torch.from_numpy(B).cuda()
            Bbuf = torch.zeros(A.nc * nv + 8, device="cuda")
            Cbuf = torch.zeros(A.nr * nv + 8, device="cuda")
            Bo, Co = Bbuf[4:4 + A.nc * nv], Cbuf[4:4 + A.nr * nv]
            assert Ba.data_ptr() % 32 == 0
            assert Bo.data_ptr() % 32 == 16 and Co.data_ptr() % 32 == 16
            Bo.copy_(Ba)
            ref = None
            for lanes in (0, 32, 16, 8):   # library tile width, then 128 / 64 / 32 columns
                if lanes and nv % (4 * lanes):
                    continue
                cfg = D.Config(alg=int(D.Alg.CSR_BALANCED), lanes_col=lanes, chunk=96)
                Ca = torch.full((A.nr * nv,), float("nan"), device="cuda")
                D.spmm(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, dA, Ba, Ca, nv=nv, cfg=cfg)
                if ref is None:
                    D.spmm(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, dA, Bo, Co, nv=nv, cfg=cfg)
                    torch.cuda.synchronize()
                    ref = Co.clone()
                    _check(A, 0, nv, B, ref.cpu().numpy(), what=f"32-lane nv={nv}")
                torch.cuda.synchronize()
                assert torch.equal(Ca, ref), \
                    f"nr={A.nr} nv={nv} lanes_col={lanes}: the window kernels differ"
