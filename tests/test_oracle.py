"""The oracle, pinned: its restatement of the reference's host code must give
exactly the reference's own outputs (committed golden fixtures, generated by
running the unmodified reference, tests/golden/make_golden.py), and, where
the reference harness is built here, match it live on more inputs."""
import os

import numpy as np
import pytest

from oracle import oracle as O


def test_known_answers(golden_dir):
    k = np.load(os.path.join(golden_dir, "golden_known.npz"))
    # values quoted from a hand run of the reference's host harness
    np.testing.assert_array_equal(k["rp_a"], [0, 0, 2, 2, 3, 3])
    np.testing.assert_array_equal(k["rp_b"], [0, 3, 3, 4, 4])
    np.testing.assert_array_equal(k["k_C_rm"], [201, 2010, 300, 3000])
    np.testing.assert_array_equal(k["k_C_cm"], [21, 30, 2100, 3000])
    np.testing.assert_array_equal(O.coo_to_csr(5, k["rp_a_rowidx"]), k["rp_a"])
    np.testing.assert_array_equal(O.coo_to_csr(4, k["rp_b_rowidx"]), k["rp_b"])
    for lay, tag in ((0, "rm"), (1, "cm")):
        C = O.spmm_f32(lay, 2, 2, k["k_rowPtr"], k["k_colIdx"], k["k_values"], k[f"k_B_{tag}"], 2)
        np.testing.assert_array_equal(C, k[f"k_C_{tag}"])


def test_rowptr_matches_reference_goldens(golden_dir):
    g = np.load(os.path.join(golden_dir, "golden_rowptr.npz"))
    n = len([x for x in g.files if x.startswith("nr_")])
    assert n >= 10
    for i in range(n):
        nr = int(g[f"nr_{i}"][0])
        np.testing.assert_array_equal(O.coo_to_csr(nr, g[f"rowIdx_{i}"]), g[f"rowPtr_{i}"])


def test_rowptr_empty_matrix_defined():
    # the reference reads rowIdx[0] unguarded (spmvspmm_benchmark.cu:44); the
    # restatement defines nnz == 0 as all-zero row pointers
    np.testing.assert_array_equal(O.coo_to_csr(4, np.zeros(0, np.int32)), [0, 0, 0, 0, 0])
    with pytest.raises(ValueError):
        O.coo_to_csr(3, [2, 1])          # unsorted
    with pytest.raises(ValueError):
        O.coo_to_csr(3, [0, 3])          # row out of range


def test_spmm_f32_bit_exact_vs_reference_goldens(golden_dir):
    """The restated host loop reproduces cpuSpmvReference bit for bit."""
    g = np.load(os.path.join(golden_dir, "golden_spmm.npz"))
    names = sorted({f.split("_")[0] for f in g.files})
    assert set(names) == {"uniform", "powerlaw", "ragged"}
    checked = 0
    for name in names:
        nr, nc = (int(x) for x in g[f"{name}_dims"])
        rp, ci, va, B = (g[f"{name}_{x}"] for x in ("rowPtr", "colIdx", "values", "B"))
        for f in g.files:
            if not f.startswith(f"{name}_C_"):
                continue
            _, _, tag, nv = f.split("_")
            nv = int(nv)
            lay = 0 if tag == "rm" else 1
            C = O.spmm_f32(lay, nr, nc, rp, ci, va, B[: nc * nv], nv)
            np.testing.assert_array_equal(C, g[f], err_msg=f)
            checked += 1
    assert checked == 3 * 7 * 2


def test_fp64_oracle_agrees_with_fp32_within_bound(golden_dir):
    g = np.load(os.path.join(golden_dir, "golden_spmm.npz"))
    nr, nc = (int(x) for x in g["powerlaw_dims"])
    rp, ci, va, B = (g[f"powerlaw_{x}"] for x in ("rowPtr", "colIdx", "values", "B"))
    for lay, tag in ((0, "rm"), (1, "cm")):
        C64, A = O.spmm_f64(lay, nr, nc, rp, ci, va, B[: nc * 32], 32)
        assert O.rel_err(g[f"powerlaw_C_{tag}_32"], C64, A) <= O.REL_TOL_F32


def test_check_result_semantics():
    ref = np.array([1.0, 2.0, 3.0, 4.0], np.float32)        # 2x2, row-major
    ok, _ = O.check_result(0, 0, 2, 2, ref, ref + 5e-4)
    assert ok
    out = ref.copy()
    out[3] += 2e-3
    ok, bad = O.check_result(0, 0, 2, 2, ref, out)
    assert not ok and bad == (1, 1)
    # col-major device output of the same matrix
    out_cm = np.array([1.0, 3.0, 2.0, 4.0], np.float32)
    ok, _ = O.check_result(0, 1, 2, 2, ref, out_cm)
    assert ok
    out = ref.copy()
    out[0] = np.nan
    assert not O.check_result(0, 0, 2, 2, ref, out)[0]


def test_calc_max_nv():
    # 80 GiB device, 1M x 1M with 10M nonzeros -> 128 fits
    assert O.calc_max_nv(1 << 20, 1 << 20, 10_000_000, 80 << 30) == 128
    # tiny memory forces halving
    mem = (1001 + 2000) * 4 + 1000 * 4 + 4 * (1000 + 1000) * 8
    assert O.calc_max_nv(1000, 1000, 1000, mem) == 8
    assert O.calc_max_nv(1000, 1000, 1000, 100) == 0


def test_partition_tables_internally_consistent():
    import daspmm as D
    for seed in range(3):
        A = D.gen_powerlaw(2000, dmax=400, seed=seed)
        for chunk, snap in ((32, 16), (128, 64), (7, 3), (1000, 1)):
            meta = O.balanced_partition(A.nr, A.rowPtr, chunk, snap).reshape(-1, 2)
            k = meta[:, 0]
            assert k[0] == 0 and k[-1] == A.nnz and meta[-1, 1] == A.nr
            assert (np.diff(k) >= 0).all()
            for c in range(1, len(meta) - 1):
                s = meta[c, 1]
                assert A.rowPtr[s] <= k[c] < A.rowPtr[s + 1]
                nominal = c * chunk
                if k[c] != nominal:   # snapped only inside a short row
                    assert k[c] == A.rowPtr[s] and A.rowPtr[s + 1] - A.rowPtr[s] < snap
            own = O.balanced_ownership(A.nr, A.rowPtr, chunk, snap).reshape(-1, 2)
            assert (own[:, 0] >= 0).all() and (own[:, 1] >= 1).all()
            lens = np.diff(A.rowPtr)
            assert (own[lens < snap, 1] == 1).all()     # short rows never split
        own = O.coo_ownership(A.nr, A.rowIdx, 64).reshape(-1, 2)
        lens = np.diff(A.rowPtr)
        assert ((own[:, 1] > 0) == (lens > 0)).all()


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built here")
def test_oracle_matches_live_reference_random_cases():
    """More inputs than the fixtures: the restatement vs the reference itself."""
    import daspmm as D
    R = O.ref()
    rng = np.random.default_rng(0)
    for t in range(12):
        A = D.gen_powerlaw(int(rng.integers(1, 400)), dmax=64, seed=t)
        nv = int(rng.choice([1, 2, 3, 5, 8, 16]))
        B = rng.uniform(-1, 1, A.nc * nv).astype(np.float32)
        for lay in (0, 1):
            ours = O.spmm_f32(lay, A.nr, A.nc, A.rowPtr, A.colIdx, A.values, B, nv)
            theirs = np.zeros(A.nr * nv, np.float32)
            R.ref_cpu_spmm(lay, A.nr, A.nc, A.nnz, nv, O._p(A.rowPtr), O._p(A.colIdx),
                           O._p(A.values), O._p(B), O._p(theirs))
            np.testing.assert_array_equal(ours, theirs)
        if A.nnz:
            rp = np.zeros(A.nr + 1, np.int32)
            ri = A.rowIdx
            R.ref_coo_to_csr(A.nr, ri.size, O._p(ri), O._p(rp))
            np.testing.assert_array_equal(O.coo_to_csr(A.nr, ri), rp)


def test_quantization_known_values():
    x = np.array([1.0, -2.5, 3.14159, 1e-3, 448.0, 500.0, -1e9, 0.0], np.float32)
    bf = O.dequantize(1, O.quantize(1, x))
    assert bf[0] == 1.0 and bf[1] == -2.5 and abs(bf[2] - 3.140625) < 1e-12
    h = O.dequantize(2, O.quantize(2, x))
    assert h[2] == np.float64(np.float16(3.14159))
    e = O.dequantize(3, O.quantize(3, x))
    assert e[0] == 1.0 and e[1] == -2.5 and e[4] == 448.0 and e[5] == 448.0 and e[6] == -448.0
    assert e[2] == 3.25  # e4m3 grid near pi: 3.0, 3.25
    # every e4m3 code round-trips
    codes = np.arange(256, dtype=np.uint8)
    vals = O.dequantize(3, codes)
    fin = ~np.isnan(vals)
    back = O.quantize(3, vals[fin].astype(np.float32))
    np.testing.assert_array_equal(O.dequantize(3, back), vals[fin])
