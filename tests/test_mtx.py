"""Matrix Market input (daspmm_mtx_info / daspmm_mtx_read), on the CPU.

Pinned to the reference: the golden file golden_mtx.npz holds what the
UNMODIFIED reference's readMtx (util/spmatrix.hpp:286-333) returns for each
fixture in tests/golden/mtx (generated by tests/golden/make_mtx.py).  The
(row, col) structure must match it exactly; values must match the oracle's
restatement, which keeps each value with its own (row, col) -- the reference
misplaces values of symmetric files after the first dropped entry, and the
test shows that on the golden data.
"""
import os

import numpy as np
import pytest

import daspmm as D
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
MTX = os.path.join(HERE, "golden", "mtx")
NAMES = sorted(n[:-4] for n in os.listdir(MTX) if n.endswith(".mtx"))


def _coo(A):
    return np.repeat(np.arange(A.nr, dtype=np.int32), np.diff(A.rowPtr)), A.colIdx


@pytest.mark.parametrize("name", NAMES)
def test_structure_matches_reference_golden(golden_dir, name):
    g = np.load(os.path.join(golden_dir, "golden_mtx.npz"))
    A = D.read_mtx(os.path.join(MTX, name + ".mtx"))
    assert [A.nr, A.nc] == list(g[name + "__shape"])
    r, c = _coo(A)
    assert np.array_equal(r, g[name + "__rows"])
    assert np.array_equal(c, g[name + "__cols"])
    nr, nc, orow, ocol, oval = O.read_mtx(os.path.join(MTX, name + ".mtx"))
    assert np.array_equal(r, orow) and np.array_equal(c, ocol)
    assert np.array_equal(A.values, oval)
    h = D.mtx_info(os.path.join(MTX, name + ".mtx"))
    assert A.nnz <= h["nnz_max"]


def test_general_values_equal_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "golden_mtx.npz"))
    for name in ("general_real", "pattern_general", "general_sparse_rows", "skew_real"):
        A = D.read_mtx(os.path.join(MTX, name + ".mtx"))
        assert np.array_equal(A.values, g[name + "__vals"]), name


def test_symmetric_values_fixed(golden_dir):
    """The reference's makeSymmetric keeps values in the pre-compaction
    order; ours keep each value at its (row, col)."""
    g = np.load(os.path.join(golden_dir, "golden_mtx.npz"))
    A = D.read_mtx(os.path.join(MTX, "symmetric_real.mtx"))
    # lower-triangle entries (2,1,-1) and (4,3,1): mirrored pairs carry those values
    dense = np.zeros((5, 5), np.float32)
    r, c = _coo(A)
    dense[r, c] = A.values
    assert dense[0, 1] == dense[1, 0] == -1.0
    assert dense[2, 3] == dense[3, 2] == 1.0
    assert dense[1, 2] == dense[2, 1] == 0.25          # first of the repeated pair
    assert np.array_equal(dense, dense.T)
    assert not np.array_equal(A.values, g["symmetric_real__vals"])   # the reference's bug


def test_keep_diagonal_and_info():
    p = os.path.join(MTX, "symmetric_real.mtx")
    A = D.read_mtx(p, keep_diagonal=True)
    dense = np.zeros((5, 5), np.float32)
    r, c = _coo(A)
    dense[r, c] = A.values
    assert dense[0, 0] == 2.0 and dense[2, 2] == 9.0 and dense[4, 4] == -3.0
    _, _, orow, ocol, oval = O.read_mtx(p, keep_diagonal=True)
    assert np.array_equal(c, ocol) and np.array_equal(A.values, oval)
    h = D.mtx_info(p)
    assert (h["nr"], h["nc"], h["entries"], h["field"], h["symmetry"], h["nnz_max"]) == \
        (5, 5, 9, 0, 1, 18)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built here")
def test_live_reference_on_seeded_files(tmp_path):
    """Larger seeded files straight through the reference's readMtx."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_mtx
    rng = np.random.default_rng(7)
    for trial, sym in enumerate(["general", "symmetric", "symmetric"]):
        n = 300
        ent = {}
        for _ in range(2500):
            r, c = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
            if sym == "symmetric" and c > r:
                r, c = c, r
            ent[(r, c)] = float(np.round(rng.uniform(-2, 2), 5))
        lst = [(r, c, v) for (r, c), v in ent.items()]
        rng.shuffle(lst)
        path = tmp_path / f"t{trial}.mtx"
        with open(path, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate real {sym}\n{n} {n} {len(lst)}\n")
            f.writelines(f"{r} {c} {v}\n" for r, c, v in lst)
        nr, nc, rr, rc, rv = make_mtx.ref_read(str(path))
        A = D.read_mtx(str(path))
        r, c = _coo(A)
        assert np.array_equal(r, rr) and np.array_equal(c, rc)
        if sym == "general":
            assert np.array_equal(A.values, rv)


def _write(tmp_path, text, name="bad.mtx"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_malformed_files(tmp_path):
    bad = [
        "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n",       # truncated
        "%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n",       # row > nr
        "%%MatrixMarket matrix coordinate real general\n3 3 1\n1 0 1.0\n",       # col < 1
        "%%MatrixMarket matrix coordinate real sideways\n3 3 0\n",               # symmetry
        "%%NotMatrixMarket matrix coordinate real general\n3 3 0\n",             # banner
        "%%MatrixMarket matrix coordinate real general\n% only comments\n",      # no size
    ]
    for i, t in enumerate(bad):
        with pytest.raises(D.DaspmmError) as ei:
            D.read_mtx(_write(tmp_path, t, f"b{i}.mtx"))
        assert ei.value.status == 9, t
    for t in ("%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1.0 2.0\n",
              "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n"):
        with pytest.raises(D.DaspmmError) as ei:
            D.read_mtx(_write(tmp_path, t, "u.mtx"))
        assert ei.value.status == 2
    with pytest.raises(D.DaspmmError):
        D.read_mtx(str(tmp_path / "missing.mtx"))
    # an empty matrix and CRLF line ends are fine
    A = D.read_mtx(_write(tmp_path, "%%MatrixMarket matrix coordinate real general\r\n"
                                    "4 2 0\r\n", "e.mtx"))
    assert A.nr == 4 and A.nnz == 0 and list(A.rowPtr) == [0] * 5
