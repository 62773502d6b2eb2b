"""The Matrix Market driver (spmvspmm_mtx): the reference's command line and
its log.csv rows (run.sh:9, spmvspmm_benchmark.cu:283-326).

Runs the driver on fixture files; it checks every variant, this library's
balanced kernel and cuSPARSE against its host loop before timing (exit code
-1 on a mismatch, as the reference), then prints one CSV row per nv.
"""
import os
import subprocess

import numpy as np
import pytest

import daspmm as D

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "da-spmmul-kernel_b200", "spmvspmm_mtx")


def _write_general(path, A):
    rows = np.repeat(np.arange(A.nr), np.diff(A.rowPtr))
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{A.nr} {A.nc} {A.nnz}\n")
        f.writelines(f"{r + 1} {c + 1} {float(v):.9g}\n" for r, c, v in zip(rows, A.colIdx, A.values))


def _run(path, *extra):
    p = subprocess.run([DRIVER, path, *extra], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [line.split(",") for line in p.stdout.strip().splitlines()]


def test_header_matches_run_sh():
    out = subprocess.run([DRIVER, "--header"], capture_output=True, text=True).stdout.strip()
    assert out.split(",")[:2] == ["filename", "KDense"] and len(out.split(",")) == 20


@pytest.mark.parametrize("which", ["generated", "symmetric_seeded"])
def test_csv_rows(cuda, tmp_path, which):
    if which == "generated":
        path = str(tmp_path / "pl.mtx")
        _write_general(path, D.gen_powerlaw(3000, dmax=300, seed=2))
    else:
        path = os.path.join(HERE, "golden", "mtx", "symmetric_seeded.mtx")
    rows = _run(path, "--with-balanced")
    nvs = [int(r[1]) for r in rows]
    assert nvs == [1, 2, 4, 8, 16, 32, 64, 128]
    for r in rows:
        assert r[0] == path
        ncus = 4 if r[1] == "1" else 10
        assert len(r) == 2 + 8 + ncus + 1
        ours = [float(x) for x in r[2:10]] + [float(r[-1])]
        assert all(v > 0 and np.isfinite(v) for v in ours), r
        cus = [float(x) for x in r[10:10 + ncus]]
        assert sum(np.isfinite(cus)) >= 2, r


def test_bad_file_fails(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")
    r = subprocess.run([DRIVER, str(p)], capture_output=True, text=True)
    assert r.returncode != 0 and "malformed" in r.stderr
