"""Batched SpMM (one persistent launch for many problems) on the GPU.

Each instance is checked against the oracle with the rules every other test
uses (FP32: the reference's 1e-3 rule and 2e-5 relative to sum|a||b|;
reduced storage: 2e-5 against FP64 of the dequantized inputs), results are
bit-identical alone and inside a batch, and a captured CUDA graph replays
the same results.
"""
import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _instances(rng, nv, n=24):
    mats = []
    for i in range(n):
        kind = i % 4
        if kind == 0:
            A = D.gen_powerlaw(int(rng.integers(100, 3000)), dmax=int(rng.integers(10, 800)),
                               seed=i)
        elif kind == 1:
            A = D.gen_random(int(rng.integers(50, 2000)), int(rng.integers(50, 2000)),
                             float(rng.uniform(0.5, 10)), seed=i)
        elif kind == 2:
            nr = int(rng.integers(1, 1500))
            A = D.gen_uniform(nr, int(rng.integers(64, 1500)), int(rng.integers(1, 40)), seed=i)
        else:  # a hub row longer than several tiles, empty leading / trailing rows
            lens = rng.integers(0, 4, 200)
            lens[:3] = 0
            lens[-5:] = 0
            lens[60] = int(rng.integers(600, 2000))
            rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
            ci = np.concatenate([np.sort(rng.choice(2500, int(k), replace=False)) for k in lens]
                                ).astype(np.int32)
            A = D.Csr(200, 2500, rp, ci, rng.uniform(-1, 1, int(rp[-1])).astype(np.float32))
        mats.append(A)
    mats.append(D.Csr(7, 9, np.zeros(8, np.int32), np.zeros(0, np.int32),
                      np.zeros(0, np.float32)))   # no nonzeros: C = beta*C
    return mats


def _prepare(mats, nv, vf, bf, rng, beta=0.0):
    import torch
    out = []
    for A in mats:
        dA = D.DeviceCsr(A)
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        Bt = torch.from_numpy(B).cuda()
        vt = dA.values
        v64 = A.values.astype(np.float64)
        if vf == D.Fmt.BF16:
            vt = D.quantize(dA.values, vf) if A.nnz else torch.zeros(1, dtype=torch.bfloat16,
                                                                     device="cuda")
            v64 = O.dequantize(1, vt.cpu().view(torch.int16).numpy().view(np.uint16))[: A.nnz]
        scales = None
        if bf == D.Fmt.F32:
            bq, b64 = Bt, B.astype(np.float64)
        elif bf == D.Fmt.BF16:
            bq = D.quantize(Bt, bf)
            b64 = O.dequantize(1, bq.cpu().view(torch.int16).numpy().view(np.uint16))
        else:
            scales = D.e4m3_scales(Bt, A.nc, nv)
            bq = D.quantize(Bt, bf, scales, nv)
            b64 = (O.dequantize(3, bq.cpu().numpy()).reshape(A.nc, nv)
                   * scales.cpu().numpy().astype(np.float64)).reshape(-1)
        C0 = rng.uniform(-1, 1, A.nr * nv).astype(np.float32)
        C = torch.from_numpy(C0.copy()).cuda()
        out.append(dict(A=dA, host=A, values=vt, val_fmt=vf, B=bq, b_fmt=bf, b_scales=scales,
                        C=C, C0=C0, nv=nv, beta=beta, v64=v64, b64=b64))
    return out


def _check(d):
    A, nv = d["host"], d["nv"]
    got = d["C"].cpu().numpy()
    c64, absc = O.spmm_f64d(0, A.nr, A.nc, A.rowPtr, A.colIdx, d["v64"], d["b64"], nv)
    if d["beta"] != 0.0:
        c64 = c64 + d["beta"] * d["C0"].astype(np.float64)
        absc = absc + abs(d["beta"]) * np.abs(d["C0"].astype(np.float64))
    e = O.rel_err(got, c64, absc)
    assert e <= O.REL_TOL_F32, f"nr={A.nr} nnz={A.nnz} nv={nv}: rel err {e}"
    if d["val_fmt"] == D.Fmt.F32 and d["b_fmt"] == D.Fmt.F32 and d["beta"] == 0.0:
        ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values,
                         d["B"].cpu().numpy(), nv)
        assert O.check_result(0, 0, A.nr, nv, ref, got)[0]


@pytest.mark.parametrize("vf,bf", [(D.Fmt.F32, D.Fmt.F32), (D.Fmt.BF16, D.Fmt.BF16),
                                   (D.Fmt.F32, D.Fmt.BF16), (D.Fmt.BF16, D.Fmt.E4M3)])
@pytest.mark.parametrize("nv", [16, 64, 96, 128])
def test_batch_parity(cuda, vf, bf, nv):
    import torch
    rng = np.random.default_rng(nv)
    mats = _instances(rng, nv)
    beta = 0.0 if nv != 96 else 0.5
    inst = _prepare(mats, nv, vf, bf, rng, beta=beta)
    b = D.Batch(inst, chunk=97)
    b.run()
    torch.cuda.synchronize()
    for d in inst:
        _check(d)
    b.close()


def test_alone_equals_in_the_mix_and_graph_replay(cuda):
    import torch
    rng = np.random.default_rng(7)
    nv = 64
    mats = _instances(rng, nv, n=16)
    inst = _prepare(mats, nv, D.Fmt.BF16, D.Fmt.BF16, rng)
    for d in inst:
        d["C"].zero_()
    batch = D.Batch(inst)
    batch.run()
    torch.cuda.synchronize()
    mixed = [d["C"].clone() for d in inst]
    for d, m in zip(inst, mixed):        # the same instance alone in its own batch
        d["C"].zero_()
        alone = D.Batch([d])
        alone.run()
        torch.cuda.synchronize()
        assert torch.equal(d["C"], m), "result differs alone vs in the batch"
        alone.close()
    s = torch.cuda.Stream()
    for d in inst:
        d["C"].zero_()
    batch.capture(s)
    for _ in range(2):                   # replays give the same results
        batch.replay(s)
        s.synchronize()
        for d, m in zip(inst, mixed):
            assert torch.equal(d["C"], m)
    items, nnz = batch.info()
    assert nnz == sum(m.nnz for m in mats) and items > len(mats)
    batch.close()


def test_batch_tune_and_autotuner(cuda, tmp_path):
    """The batch row-tile tuner returns one of its candidates; the SpMM
    autotuner caches a choice that DASPMM_ALG_AUTO then uses, and the cache
    survives a save / load round trip."""
    import torch
    rng = np.random.default_rng(3)
    mats = _instances(rng, 64, n=8)
    inst = _prepare(mats, 64, D.Fmt.F32, D.Fmt.BF16, rng)
    best, us = D.Batch.tune(inst, chunks=[64, 256], reps=2)
    assert best in (64, 256) and us > 0
    A = D.gen_powerlaw(20000, seed=4)
    dA = D.DeviceCsr(A)
    B = torch.from_numpy(D.gen_dense(A.nc * 128, seed=2)).cuda()
    C = torch.zeros(A.nr * 128, device="cuda")
    fp = D.fingerprint(0, dA, 128)
    lens = np.diff(A.rowPtr)
    assert fp["max_row"] == lens.max() and fp["nnz"] == A.nnz
    assert fp["p50"] >= np.percentile(lens, 50) - 1e-9 and fp["p99"] <= lens.max()
    cfg, us = D.autotune(0, dA, B, C, 128, reps=2)
    assert us > 0
    auto = D.default_config(D.Alg.AUTO, 0, A.nr, A.nc, A.nnz, 128)
    assert auto.as_dict() == cfg.as_dict()
    C.zero_()
    D.spmm(D.Alg.AUTO, 0, dA, B, C, nv=128)
    torch.cuda.synchronize()
    ref = O.spmm_f32(0, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B.cpu().numpy(), 128)
    assert O.check_result(0, 0, A.nr, 128, ref, C.cpu().numpy())[0]
    path = str(tmp_path / "tune.txt")
    assert D.lib().daspmm_tune_save(path.encode()) == 0
    D.lib().daspmm_tune_clear()
    assert D.default_config(D.Alg.AUTO, 0, A.nr, A.nc, A.nnz, 128).as_dict() != cfg.as_dict() \
        or cfg.alg == 4
    assert D.lib().daspmm_tune_load(path.encode()) == 0
    assert D.default_config(D.Alg.AUTO, 0, A.nr, A.nc, A.nnz, 128).as_dict() == cfg.as_dict()


def test_batch_tile_width_and_joint_tuner(cuda):
    """Narrower column tiles (lanes_col 16 / 8: at most 64 / 32 floats) give
    bit-identical results (each output element is summed in the same order
    whatever the tile), and the joint row-tile / column-tile tuner returns one
    of its candidates."""
    import torch
    rng = np.random.default_rng(11)
    nv = 128
    mats = _instances(rng, nv, n=12)
    for vf, bf in ((D.Fmt.F32, D.Fmt.F32), (D.Fmt.F32, D.Fmt.BF16)):
        inst = _prepare(mats, nv, vf, bf, rng)
        ref = None
        for lanes in (0, 16, 8):
            for d in inst:
                d["C"].fill_(float("nan"))
            b = D.Batch(inst, chunk=256, lanes_col=lanes)
            b.run()
            torch.cuda.synchronize()
            out = [d["C"].clone() for d in inst]
            b.close()
            if ref is None:
                ref = out
                for d in inst:
                    _check(d)
            else:
                for r, o in zip(ref, out):
                    assert torch.equal(r, o), f"lanes_col {lanes} differs"
        best, us = D.Batch.tune_ex(inst, chunks=[128, 512], widths=[128, 64], reps=2)
        assert best.chunk in (128, 512) and best.lanes_col in (32, 16) and us > 0
    with pytest.raises(D.DaspmmError):
        D.Batch(inst, lanes_col=4)


def _offset(t):
    """A copy of t 16 bytes past a 32-byte boundary, with the buffer that
    holds it (keep both alive)."""
    import torch
    eb = t.element_size()
    buf = torch.empty(t.numel() + 64 // eb, dtype=t.dtype, device="cuda")
    v = buf[16 // eb: 16 // eb + t.numel()]
    v.copy_(t)
    assert v.data_ptr() % 32 == 16
    return v, buf


@pytest.mark.parametrize("vf,bf", [(D.Fmt.F32, D.Fmt.F32), (D.Fmt.F32, D.Fmt.BF16),
                                   (D.Fmt.BF16, D.Fmt.E4M3)])
def test_group_gather_equals_32_lane(cuda, vf, bf):
    """Runs of whole rows and pieces of long rows take the worker-group
    gather when B and C are 32-byte aligned and the 32-lane one when they are
    16 bytes off: the same sums in the same order, so the batches' C are
    bit-identical (small tiles: the hub rows are cut into many pieces)."""
    import torch
    rng = np.random.default_rng(19)
    for nv in (32, 64, 128):
        mats = _instances(rng, nv, n=12)
        inst = _prepare(mats, nv, vf, bf, rng)
        off, keep = [], []
        for d in inst:
            e = dict(d)
            e["B"], kb = _offset(d["B"])
            e["C"], kc = _offset(d["C"])
            keep += [kb, kc]
            off.append(e)
        outs = []
        for group in (inst, off):
            for d in group:
                d["C"].fill_(float("nan"))
            b = D.Batch(group, chunk=97)
            b.run()
            torch.cuda.synchronize()
            outs.append([d["C"].clone() for d in group])
            b.close()
        for d, x, y in zip(inst, *outs):
            assert torch.equal(x, y), f"nv={nv} nr={d['host'].nr}: the gathers differ"
        for d, x in zip(inst, outs[0]):
            d["C"].copy_(x)
            _check(d)
