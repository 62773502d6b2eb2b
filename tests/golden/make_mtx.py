"""Matrix Market fixtures and the reference's readMtx output on them.

Writes small .mtx files into tests/golden/mtx/ (seeded, hand-shaped to hit
every case readMtx handles: general real with repeated pairs and comments,
symmetric real with diagonal entries and a repeated pair, pattern, integer,
skew-symmetric, empty rows) and, when the reference tree is mounted, stores
what the UNMODIFIED reference's readMtx<float> (util/spmatrix.hpp:286-333,
makeSymmetric included) returns for each, as (rows, cols, values) in its
output order, in golden_mtx.npz.

Run (needs the reference tree, so only where it is mounted):
    make -C oracle && python tests/golden/make_mtx.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "da-spmmul-kernel_b200"))

from oracle import oracle as O  # noqa: E402

MTX = os.path.join(HERE, "mtx")


def _write(name, field, sym, nr, nc, entries, comments=("",)):
    lines = [f"%%MatrixMarket matrix coordinate {field} {sym}"]
    lines += [f"%{c}" for c in comments]
    lines.append(f"{nr} {nc} {len(entries)}")
    for e in entries:
        if field == "pattern":
            lines.append(f"{e[0]} {e[1]}")
        elif field == "integer":
            lines.append(f"{e[0]} {e[1]} {int(e[2])}")
        else:
            lines.append(f"{e[0]} {e[1]} {e[2]:.6g}")
    with open(os.path.join(MTX, name), "w") as f:
        f.write("\n".join(lines) + "\n")


def fixtures():
    rng = np.random.default_rng(2022)
    os.makedirs(MTX, exist_ok=True)
    # general: unsorted, a repeated pair, an empty leading and trailing row
    ent = [(3, 2, 1.5), (2, 4, -2.25), (2, 1, 0.5), (3, 2, 4.0), (5, 5, 3.0), (2, 2, 7.0)]
    _write("general_real.mtx", "real", "general", 6, 5, ent, ("comment one", "", " x"))
    # symmetric: lower triangle with diagonal entries and one repeated pair
    ent = [(1, 1, 2.0), (2, 1, -1.0), (3, 2, 0.25), (3, 3, 9.0), (4, 1, 5.5), (4, 3, 1.0),
           (3, 2, 0.75), (5, 5, -3.0), (5, 4, 6.0)]
    _write("symmetric_real.mtx", "real", "symmetric", 5, 5, ent)
    # symmetric, seeded: 40x40 lower triangle with ~25% of the diagonal
    ent = []
    for r in range(1, 41):
        for c in range(1, r + 1):
            if (r == c and rng.random() < 0.25) or (r != c and rng.random() < 0.12):
                ent.append((r, c, float(np.round(rng.uniform(-1, 1), 4))))
    rng.shuffle(ent)
    _write("symmetric_seeded.mtx", "real", "symmetric", 40, 40, [tuple(e) for e in ent])
    # pattern general
    ent = sorted({(int(rng.integers(1, 31)), int(rng.integers(1, 21))) for _ in range(60)})
    rng.shuffle(ent)
    _write("pattern_general.mtx", "pattern", "general", 30, 20, ent)
    # integer symmetric (no repeated pairs)
    ent = [(1, 1, 4), (2, 1, -2), (3, 1, 7), (3, 3, 1), (4, 2, 3)]
    _write("integer_symmetric.mtx", "integer", "symmetric", 4, 4, ent)
    # skew-symmetric: read as stored (the reference does not mirror it)
    ent = [(2, 1, 1.0), (3, 1, -2.0), (3, 2, 0.5)]
    _write("skew_real.mtx", "real", "skew-symmetric", 3, 3, ent)
    # general with many empty rows and one full row
    ent = [(7, c, float(c) / 8) for c in range(1, 9)] + [(2, 3, -1.0)]
    _write("general_sparse_rows.mtx", "real", "general", 12, 8, ent)


def ref_read(path, cap=100000):
    import ctypes
    R = O.ref()
    f = R.ref_read_mtx
    f.restype = ctypes.c_int
    nr, nc = ctypes.c_int(), ctypes.c_int()
    rows = np.zeros(cap, np.int32)
    cols = np.zeros(cap, np.int32)
    vals = np.zeros(cap, np.float32)
    n = f(path.encode(), ctypes.byref(nr), ctypes.byref(nc), cap, O._p(rows), O._p(cols),
          O._p(vals))
    assert n >= 0
    return nr.value, nc.value, rows[:n].copy(), cols[:n].copy(), vals[:n].copy()


def main():
    fixtures()
    if not O.ref_available():
        print("reference harness not built: fixtures written, golden_mtx.npz unchanged")
        return
    out = {}
    for name in sorted(os.listdir(MTX)):
        nr, nc, r, c, v = ref_read(os.path.join(MTX, name))
        key = name[:-4]
        out[f"{key}__shape"] = np.array([nr, nc], np.int32)
        out[f"{key}__rows"] = r
        out[f"{key}__cols"] = c
        out[f"{key}__vals"] = v
    np.savez_compressed(os.path.join(HERE, "golden_mtx.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_mtx.npz"), len(out) // 4, "matrices")


if __name__ == "__main__":
    main()
