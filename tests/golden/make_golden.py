"""Generate the golden fixtures in this directory from the UNMODIFIED reference.

The reference (ASPLOS-2022/DA-SpMMul-kernel) ships no tests, matrices or
golden vectors.  Its only correctness rule is the host loop cpuSpmvReference
(spmvspmm_benchmark.cu:11-39) with the absolute 1e-3 check (:93-116), and
its COO->CSR build generateCsrRowPtrArray (:41-76).  This script runs those
functions themselves -- compiled from the reference tree by oracle/Makefile into
oracle/_ref/libref.so -- on seeded inputs and stores inputs and outputs:

  golden_known.npz   hand-checkable known answers (2x2 products, row pointers)
  golden_rowptr.npz  generateCsrRowPtrArray on row lists with empty leading,
                     middle and trailing rows
  golden_spmm.npz    cpuSpmvReference outputs, both layouts, nv in
                     {1,2,3,4,8,16,32} on three seeded matrices

Run (needs the reference tree, so only where it is mounted):
    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "da-spmmul-kernel_b200"))

from oracle import oracle as O  # noqa: E402

NVS = [1, 2, 3, 4, 8, 16, 32]


def ref_spmm(layout, nr, nc, rp, ci, va, B, nv):
    R = O.ref()
    C = np.zeros(nr * nv, np.float32)
    rp, ci, va, B = (np.ascontiguousarray(x) for x in (rp, ci, va, B))
    R.ref_cpu_spmm(layout, nr, nc, int(rp[-1]), nv, O._p(rp), O._p(ci), O._p(va), O._p(B),
                   O._p(C))
    return C


def ref_rowptr(nr, rowIdx):
    ri = np.ascontiguousarray(rowIdx, np.int32)
    rp = np.zeros(nr + 1, np.int32)
    assert O.ref().ref_coo_to_csr(nr, ri.size, O._p(ri), O._p(rp)) == 0
    return rp


def matrices():
    import daspmm as D
    rng = np.random.default_rng(12345)
    out = {}
    A = D.gen_uniform(64, 48, 5, seed=3)
    out["uniform"] = (A.nr, A.nc, A.rowPtr, A.colIdx, A.values)
    A = D.gen_powerlaw(300, dmax=120, seed=5)
    out["powerlaw"] = (A.nr, A.nc, A.rowPtr, A.colIdx, A.values)
    # rows with empty leading / middle / trailing runs and one long row
    nr, nc = 40, 37
    lens = rng.integers(0, 6, nr)
    lens[:3] = 0
    lens[17:20] = 0
    lens[-4:] = 0
    lens[25] = 33
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(nc, int(k), replace=False)) for k in lens]
                        ).astype(np.int32)
    va = rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)
    out["ragged"] = (nr, nc, rp, ci, va)
    return out


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/libref.so is missing: run `make -C oracle` where the "
                 "reference tree is mounted")
    # known answers
    known = {}
    known["rp_a_rowidx"] = np.array([1, 1, 3], np.int32)
    known["rp_a"] = ref_rowptr(5, known["rp_a_rowidx"])
    known["rp_b_rowidx"] = np.array([0, 0, 0, 2], np.int32)
    known["rp_b"] = ref_rowptr(4, known["rp_b_rowidx"])
    rp = np.array([0, 2, 3], np.int32)
    ci = np.array([0, 1, 1], np.int32)
    va = np.array([1, 2, 3], np.float32)
    known["k_rowPtr"], known["k_colIdx"], known["k_values"] = rp, ci, va
    known["k_B_rm"] = np.array([1, 10, 100, 1000], np.float32)
    known["k_C_rm"] = ref_spmm(0, 2, 2, rp, ci, va, known["k_B_rm"], 2)
    known["k_B_cm"] = np.array([1, 10, 100, 1000], np.float32)
    known["k_C_cm"] = ref_spmm(1, 2, 2, rp, ci, va, known["k_B_cm"], 2)
    np.savez_compressed(os.path.join(HERE, "golden_known.npz"), **known)

    # row pointers
    rng = np.random.default_rng(7)
    rpz = {}
    cases = [(6, [0, 0, 5, 5]), (10, [2, 2, 2, 9]), (3, [0, 1, 2]), (8, [7]),
             (1, [0, 0, 0])]
    for t in range(6):
        nr = int(rng.integers(1, 60))
        cases.append((nr, np.sort(rng.integers(0, nr, int(rng.integers(1, 200))))))
    for i, (nr, ri) in enumerate(cases):
        ri = np.asarray(ri, np.int32)
        rpz[f"nr_{i}"] = np.array([nr], np.int32)
        rpz[f"rowIdx_{i}"] = ri
        rpz[f"rowPtr_{i}"] = ref_rowptr(nr, ri)
    np.savez_compressed(os.path.join(HERE, "golden_rowptr.npz"), **rpz)

    # SpMM outputs
    sp = {}
    for name, (nr, nc, rp, ci, va) in matrices().items():
        sp[f"{name}_dims"] = np.array([nr, nc], np.int32)
        sp[f"{name}_rowPtr"], sp[f"{name}_colIdx"], sp[f"{name}_values"] = rp, ci, va
        brng = np.random.default_rng(99)
        Bmax = brng.uniform(-1, 1, nc * max(NVS)).astype(np.float32)
        sp[f"{name}_B"] = Bmax
        for nv in NVS:
            B = Bmax[: nc * nv]
            for lay, tag in ((0, "rm"), (1, "cm")):
                sp[f"{name}_C_{tag}_{nv}"] = ref_spmm(lay, nr, nc, rp, ci, va, B, nv)
    np.savez_compressed(os.path.join(HERE, "golden_spmm.npz"), **sp)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
