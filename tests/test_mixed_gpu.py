"""Mixed precision on the GPU: BF16 / FP16 storage, FP8 E4M3 B with per-column
FP32 scales, FP32 accumulation, Kahan rows.

Error statements (FP64 oracle, oracle/oracle.c):
  * against FP64 of the quantized (dequantized) inputs -- the kernel's own
    arithmetic -- per element, relative to sum_p |a_p||b_p|: <= 2e-5, the FP32
    bound of every other test;
  * against FP64 of the original FP32 inputs -- storage + arithmetic -- as
    max |c - c64| / max sum|a||b| (oracle.rel_err_max): <= 1e-2 for BF16 and
    FP16 storage, <= 2^-4 for E4M3 B (its 3-bit mantissa rounds by up to 2^-4).
Quantization is bit-exact with the oracle's round-to-nearest-even.
"""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

COMBOS = [(D.Fmt.BF16, D.Fmt.BF16), (D.Fmt.F16, D.Fmt.F16), (D.Fmt.F32, D.Fmt.E4M3),
          (D.Fmt.BF16, D.Fmt.E4M3), (D.Fmt.F32, D.Fmt.F32)]


def _quant_inputs(A, B, val_fmt, b_fmt, nv):
    """Device tensors for (values, B, scales) and their float64 dequantized host copies."""
    import torch
    vt = torch.from_numpy(A.values).cuda()
    Bt = torch.from_numpy(B).cuda()
    scales = None
    if val_fmt == D.Fmt.F32:
        vq, v64 = vt, A.values.astype(np.float64)
    else:
        vq = D.quantize(vt, val_fmt)
        v64 = O.dequantize(int(val_fmt), vq.cpu().view(torch.int16).numpy().view(np.uint16))
    if b_fmt == D.Fmt.F32:
        bq, b64 = Bt, B.astype(np.float64)
    elif b_fmt == D.Fmt.E4M3:
        scales = D.e4m3_scales(Bt, A.nc, nv)
        bq = D.quantize(Bt, b_fmt, scales, nv)
        sc = scales.cpu().numpy().astype(np.float64)
        b64 = (O.dequantize(3, bq.cpu().numpy()).reshape(A.nc, nv) * sc).reshape(-1)
    else:
        bq = D.quantize(Bt, b_fmt)
        b64 = O.dequantize(int(b_fmt), bq.cpu().view(torch.int16).numpy().view(np.uint16))
    return vq, bq, scales, v64, b64


def _run_mixed(A, dA, B, nv, val_fmt, b_fmt, kahan_min=0, beta=0.0, C0=None, cfg=None):
    import torch
    vq, bq, scales, v64, b64 = _quant_inputs(A, B, val_fmt, b_fmt, nv)
    C = (torch.from_numpy(C0).cuda() if C0 is not None
         else torch.full((A.nr * nv,), float("nan"), dtype=torch.float32, device="cuda"))
    if C0 is None and beta != 0.0:
        C.zero_()
    D.spmm_mixed(dA, vq, val_fmt, bq, b_fmt, C, nv, b_scales=scales, beta=beta,
                 kahan_min=kahan_min, cfg=cfg)
    torch.cuda.synchronize()
    return C.cpu().numpy(), v64, b64


def _errors(A, nv, B, C, v64, b64, beta=0.0, C0=None):
    cq, aq = O.spmm_f64d(0, A.nr, A.nc, A.rowPtr, A.colIdx, v64, b64, nv)
    c64, a64 = O.spmm_f64(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
    if beta != 0.0:
        extra = beta * C0.astype(np.float64)
        cq, c64 = cq + extra, c64 + extra
        aq, a64 = aq + np.abs(extra), a64 + np.abs(extra)
    return O.rel_err(C, cq, aq), O.rel_err_max(C, c64, a64)


def _tol(b_fmt):
    return O.E4M3_TOL if b_fmt == D.Fmt.E4M3 else O.MIXED_TOL


@pytest.fixture(scope="module")
def mats(cuda):
    rng = np.random.default_rng(14)
    lens = rng.integers(0, 5, 300)
    lens[7] = 2500
    lens[:3] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(3000, int(k), replace=False)) for k in lens]
                        ).astype(np.int32)
    va = rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)
    out = {"powerlaw": D.gen_powerlaw(4000, dmax=900, seed=3),
           "hub": D.Csr(300, 3000, rp, ci, va),
           "random": D.gen_random(700, 650, 6.0, seed=9)}
    return {k: (A, D.DeviceCsr(A)) for k, A in out.items()}


def test_quantizers_bit_exact(cuda):
    import torch
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-3, 3, 5000), rng.normal(0, 100, 3000),
                        [0.0, -0.0, 1e-30, 448.0, 449.0, 1e6, -1e6, 2 ** -10]]).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    for fmt in (D.Fmt.BF16, D.Fmt.F16):
        q = D.quantize(xt, fmt).cpu().view(torch.int16).numpy().view(np.uint16)
        np.testing.assert_array_equal(q, O.quantize(int(fmt), x), err_msg=fmt.name)
    # E4M3 with per-column scales over a 2-D matrix
    nr, nv = 500, 32
    B = (rng.normal(0, 1, (nr, nv)) * rng.uniform(0.01, 50, nv)).astype(np.float32)
    Bt = torch.from_numpy(B.reshape(-1)).cuda()
    sc = D.e4m3_scales(Bt, nr, nv).cpu().numpy()
    want_sc = np.abs(B).max(axis=0) / np.float32(448.0)
    np.testing.assert_array_equal(sc, want_sc.astype(np.float32))
    q = D.quantize(Bt, D.Fmt.E4M3, torch.from_numpy(sc).cuda(), nv).cpu().numpy()
    np.testing.assert_array_equal(q, O.quantize(3, (B / sc).astype(np.float32)))


@pytest.mark.parametrize("name", ["powerlaw", "hub", "random"])
def test_mixed_products(mats, name):
    A, dA = mats[name]
    rng = np.random.default_rng(21)
    for nv in (32, 64, 128, 256):
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        for vf, bf in COMBOS:
            for kmin in (0, 16):
                C, v64, b64 = _run_mixed(A, dA, B, nv, vf, bf, kahan_min=kmin)
                eq, e64 = _errors(A, nv, B, C, v64, b64)
                what = f"{name} nv={nv} {vf.name}/{bf.name} kahan>={kmin}"
                assert eq <= O.REL_TOL_F32, f"{what}: vs quantized-input FP64 {eq}"
                assert e64 <= _tol(bf), f"{what}: vs FP32-input FP64 {e64}"
    # beta and small chunks (hub rows split across many chunks)
    nv = 64
    B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
    C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
    cfg = D.Config(alg=4, chunk=37, snap=11)
    C, v64, b64 = _run_mixed(A, dA, B, nv, D.Fmt.BF16, D.Fmt.E4M3, beta=-0.5, C0=C0, cfg=cfg)
    eq, e64 = _errors(A, nv, B, C, v64, b64, beta=-0.5, C0=C0)
    assert eq <= O.REL_TOL_F32 and e64 <= O.E4M3_TOL


def test_kahan_reduces_error_on_a_long_row(cuda):
    """A 6000-term row whose terms cancel: compensated sums are closer to FP64."""
    import torch
    rng = np.random.default_rng(5)
    n = 6000
    big = rng.uniform(0.5, 1.0, n // 2)
    vals = np.concatenate([big, -big + rng.uniform(-1e-4, 1e-4, n // 2)])
    vals = rng.permutation(vals).astype(np.float32)
    nv = 32
    A = D.Csr(1, n, np.array([0, n], np.int32), np.arange(n, dtype=np.int32), vals)
    dA = D.DeviceCsr(A)
    B = (1.0 + rng.uniform(0, 1e-3, n * nv)).astype(np.float32)
    errs = {}
    for kmin in (0, 1000):
        C, v64, b64 = _run_mixed(A, dA, B, nv, D.Fmt.F32, D.Fmt.F32, kahan_min=kmin,
                                 cfg=D.Config(alg=4, chunk=100000))
        c64, _ = O.spmm_f64d(0, 1, n, A.rowPtr, A.colIdx, v64, b64, nv)
        errs[kmin] = float(np.abs(C - c64).max())
    assert errs[1000] <= errs[0]
    assert errs[1000] < 1e-4


def _sampled_errors(A, nv, Bt, vf, bf, vq, bq, scales, C):
    """Error statements (oracle.mixed_errors) of a device result C over the
    leading rows the FP64 oracle checks (oracle.sample_rows)."""
    import torch
    R = O.sample_rows(A.rowPtr, A.colIdx, nv)
    rp, ci, va32, cols = O.row_slice(A.rowPtr, A.colIdx, A.values, 0, R)
    colt = torch.from_numpy(cols.astype(np.int64)).cuda()
    b32 = Bt.view(A.nc, nv)[colt].cpu().numpy().reshape(-1)
    p1 = int(A.rowPtr[R])
    if vf == D.Fmt.F32:
        va64 = va32.astype(np.float64)
    else:
        va64 = O.dequantize(int(vf), vq[:p1].cpu().view(torch.int16).numpy().view(np.uint16))
    if bf == D.Fmt.F32:
        b64 = b32.astype(np.float64)
    elif bf == D.Fmt.E4M3:
        q = bq.view(A.nc, nv)[colt].cpu().numpy().reshape(-1)
        sc = scales.cpu().numpy().astype(np.float64)
        b64 = (O.dequantize(3, q).reshape(-1, nv) * sc).reshape(-1)
    else:
        q = bq.view(A.nc, nv)[colt].cpu().view(torch.int16).numpy().view(np.uint16)
        b64 = O.dequantize(int(bf), q.reshape(-1))
    return R, O.mixed_errors(rp, ci, va32, va64, b32, b64, C[: R * nv].cpu().numpy(), nv)


@pytest.mark.slow
def test_config3_full_size_error_bound(cuda):
    """The mixed-precision configuration at full size: the 262k power-law A and
    a 1M-row uniform-random A (average degree 8), N in {32, 128, 512}, values
    and B in BF16 or FP16, and BF16 values with E4M3 B (per-column scales);
    FP32 accumulation, Kahan on rows of >= 256 nonzeros.  Checked on the rows
    the FP64 oracle can hold (all of them where the product has <= 2^25
    elements, else the leading rows, oracle.sample_rows):
      * kernel arithmetic, per element against its condition scale: <= 2e-5;
      * storage + arithmetic, max-norm relative: <= 1e-2 (BF16, FP16), <= 2^-4
        (E4M3), and per element against its condition scale <= 1e-2 for
        BF16 / FP16 (each stored product is off by <= 2^-8 |a||b|)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    combos = ((D.Fmt.BF16, D.Fmt.BF16), (D.Fmt.F16, D.Fmt.F16), (D.Fmt.BF16, D.Fmt.E4M3))
    for A in (D.gen_powerlaw(262144, seed=0), D.gen_random(1 << 20, 1 << 20, 8.0, seed=0)):
        dA = D.DeviceCsr(A)
        for nv in (32, 128, 512):
            Bt = torch.empty(A.nc * nv, device="cuda").uniform_(-1, 1, generator=g)
            C = torch.empty(A.nr * nv, device="cuda")
            for vf, bf in combos:
                vq = D.quantize(dA.values, vf)
                scales = D.e4m3_scales(Bt, A.nc, nv) if bf == D.Fmt.E4M3 else None
                bq = D.quantize(Bt, bf, scales, nv if scales is not None else 0)
                C.fill_(float("nan"))
                D.spmm_mixed(dA, vq, vf, bq, bf, C, nv, b_scales=scales, kahan_min=256)
                torch.cuda.synchronize()
                R, e = _sampled_errors(A, nv, Bt, vf, bf, vq, bq, scales, C)
                what = f"nr={A.nr} nv={nv} {vf.name}/{bf.name} rows 0..{R - 1}"
                print(what, e)
                assert e["kernel"] <= O.REL_TOL_F32, what
                assert e["storage"]["norm_max"] <= _tol(bf), what
                if bf != D.Fmt.E4M3:
                    assert e["storage"]["cond_max"] <= O.MIXED_TOL, what
                del vq, bq
            del Bt, C


def test_group_kernel_equals_32_lane_kernel_mixed(mats):
    """Reduced-precision B runs the worker-group window kernel (8-byte lane
    loads for 32- and 64-column tiles, 16-byte ones for 128) when C is
    32-byte aligned, the 32-lane one when C is 16 bytes off: same chunks and
    order of summation, bit-identical C.  The hub matrix has empty rows."""
    import torch
    rng = np.random.default_rng(31)
    for name in ("powerlaw", "random", "hub"):
        A, dA = mats[name]
        for nv in (32, 64, 128, 256, 384):
            B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
            for vf, bf in ((D.Fmt.BF16, D.Fmt.BF16), (D.Fmt.F16, D.Fmt.F16),
                           (D.Fmt.BF16, D.Fmt.E4M3), (D.Fmt.F32, D.Fmt.E4M3)):
                vq, bq, scales, v64, b64 = _quant_inputs(A, B, vf, bf, nv)
                Ca = torch.full((A.nr * nv,), float("nan"), device="cuda")
                Cbuf = torch.full((A.nr * nv + 8,), float("nan"), device="cuda")
                Co = Cbuf[4:4 + A.nr * nv]
                assert Ca.data_ptr() % 32 == 0 and Co.data_ptr() % 32 == 16
                for C in (Ca, Co):
                    D.spmm_mixed(dA, vq, vf, bq, bf, C, nv, b_scales=scales)
                torch.cuda.synchronize()
                assert torch.equal(Ca, Co), f"{name} nv={nv} {vf.name}/{bf.name}"
                eq, e64 = _errors(A, nv, B, Ca.cpu().numpy(), v64, b64)
                assert eq <= O.REL_TOL_F32 and e64 <= _tol(bf)
