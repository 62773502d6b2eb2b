"""Host-side checks that need no GPU: the C-ABI library loads and exports
every symbol its public headers declare, configuration resolution, argument
errors, and the deterministic input generators."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import daspmm as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        if 'extern "C"' not in txt:   # C++ drop-in headers: templates and inlines only
            continue
        # C declarations of the ABI: "<type> daspmm_xxx(" at line start
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(daspmm_\w+)\s*\(", txt, re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert "daspmm_spmm" in names and "daspmm_compat_spmm" in names
    lib = ctypes.CDLL(D.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_abi_version_and_status_strings():
    L = D.lib()
    assert L.daspmm_abi_version() == 2
    for s in range(10):
        assert L.daspmm_status_string(s)
    assert L.daspmm_status_string(0) == b"ok"


def test_default_configs():
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, 262144, 262144, 1_227_000, 128)
    assert (c.vec, c.lanes_col, c.lanes_nnz, c.cf, c.pipe) == (4, 32, 1, 1, 4)
    assert c.chunk == 96 and c.snap == 48 and c.block == 256   # one 128-column tile
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, 262144, 262144, 1_227_000, 512)
    assert c.chunk == 128 and c.snap == 64 and c.block == 256
    # mixed precision keeps 128-nonzero chunks: never more workspace than the
    # FP32 default a caller sizes it with
    for nv in (32, 64, 128, 256, 512):
        f32 = D.workspace_bytes(D.Config(alg=4), 0, 262144, 262144, 1_227_000, nv)
        mixed = D.workspace_bytes(D.Config(alg=4, pipe=4, chunk=128), 0, 262144, 262144,
                                  1_227_000, nv)
        assert mixed <= f32, nv
    # the TMA ring sizes one wave of chunks over 148 SMs x 12 warps (no GPU here: 148)
    r = D.Config(alg=4, pipe=2)
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, 262144, 262144, 1_227_000, 128)
    assert D.workspace_bytes(r, 0, 262144, 262144, 1_227_000, 128) > 0
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.ROW_MAJOR, 1000, 1000, 9000, 30)
    assert c.pipe == 1 and c.chunk == 64           # nv % 32 != 0: register gather (V=2, L=16)
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.COL_MAJOR, 1000, 1000, 9000, 64)
    assert c.pipe == 5                             # column-major through row-major
    assert D.workspace_bytes(c, 1, 1000, 800, 9000, 64) >= (1000 + 800) * 64 * 4
    c = D.default_config(D.Alg.CSR_BALANCED, D.Layout.COL_MAJOR, 1000, 1000, 9000, 2)
    assert c.pipe == 1
    c = D.default_config(D.Alg.CSR_VECTOR, D.Layout.ROW_MAJOR, 100, 100, 1000, 1)
    assert (c.vec, c.lanes_col, c.lanes_nnz) == (1, 1, 32)
    c = D.default_config(D.Alg.CSR_SCALAR, D.Layout.ROW_MAJOR, 100, 100, 1000, 512)
    assert (c.vec, c.lanes_col, c.cf) == (4, 32, 2)
    c = D.default_config(D.Alg.COO_SCALAR, D.Layout.COL_MAJOR, 100, 100, 1000, 16)
    assert (c.vec, c.lanes_col, c.cf) == (1, 1, 8)
    c = D.default_config(D.Alg.CSR_SCALAR, D.Layout.ROW_MAJOR, 100, 100, 1000, 3)
    assert c.vec == 1 and c.lanes_col == 4


def test_invalid_arguments_rejected_before_any_device_work():
    L = D.lib()
    # bad layout / alg / nv: resolved before any CUDA call
    assert L.daspmm_spmm(0, 7, 4, 4, 4, 4, None, None, None, None, None, None, 0.0, None) == 1
    assert L.daspmm_spmm(9, 0, 4, 4, 4, 4, None, None, None, None, None, None, 0.0, None) == 1
    assert L.daspmm_spmm(0, 0, 4, 4, 4, 0, None, None, None, None, None, None, 0.0, None) == 1
    # compat returns cudaErrorInvalidValue (1) for an unknown algorithm
    assert L.daspmm_compat_spmm(7, 0, 4, 4, 4, 4, None, None, None, None, None, None) == 1
    # empty problem is a no-op
    assert L.daspmm_spmm(0, 0, 0, 4, 0, 4, None, None, None, None, None, None, 0.0, None) == 0
    cfg = D.Config(alg=2, lanes_nnz=4)   # COO scalar has S == 1
    assert L.daspmm_spmm_ex(ctypes.byref(cfg), 0, 4, 4, 4, 4, None, None, None, None, None,
                            None, 0.0, None, 0, None) == 2
    cfg = D.Config(alg=1, lanes_col=8, lanes_nnz=8)  # L*S > 32
    assert L.daspmm_spmm_ex(ctypes.byref(cfg), 0, 4, 4, 4, 8, None, None, None, None, None,
                            None, 0.0, None, 0, None) == 1


def test_workspace_bytes():
    cfg = D.default_config(D.Alg.CSR_BALANCED, 0, 1000, 1000, 10000, 64)
    nch = D.num_chunks(10000, cfg.chunk)
    assert D.workspace_bytes(cfg, 0, 1000, 1000, 10000, 64) >= nch * 2 * 64 * 4 + (nch + 1) * 8
    assert D.workspace_bytes(D.default_config(0, 0, 1000, 1000, 10000, 64), 0, 1000, 1000, 10000,
                             64) == 0
    assert D.num_chunks(0, 128) == 1 and D.num_chunks(129, 128) == 2 and D.num_chunks(5, 0) == -1


def test_generators_deterministic_and_well_formed():
    a = D.gen_uniform(200, 150, 16, seed=0)
    b = D.gen_uniform(200, 150, 16, seed=0)
    np.testing.assert_array_equal(a.colIdx, b.colIdx)
    np.testing.assert_array_equal(a.values, b.values)
    assert a.nnz == 200 * 16
    for r in range(a.nr):
        row = a.colIdx[a.rowPtr[r]:a.rowPtr[r + 1]]
        assert (np.diff(row) > 0).all() and row.min() >= 0 and row.max() < 150
    assert a.values.min() >= -1 and a.values.max() < 1
    c = D.gen_uniform(200, 150, 16, seed=1)
    assert not np.array_equal(a.colIdx, c.colIdx)

    p = D.gen_powerlaw(20000, seed=0)
    lens = np.diff(p.rowPtr)
    assert lens.min() >= 1 and lens.max() <= 4096
    assert 4.2 < lens.mean() < 5.2          # E[k] ~ 4.68 for (k+0.16)^-2.1 on [1,4096]
    for r in range(0, p.nr, 997):
        row = p.colIdx[p.rowPtr[r]:p.rowPtr[r + 1]]
        assert (np.diff(row) > 0).all()
    indeg = np.bincount(p.colIdx, minlength=p.nc)
    # preferential attachment: in-degrees far above a uniform draw (max ~ mean + 4 sd)
    assert indeg.max() > 5 * max(1.0, indeg.mean())

    q = D.gen_random(5000, 4000, 8.0, seed=2)
    lq = np.diff(q.rowPtr)
    assert 7.5 < lq.mean() < 8.5 and (lq == 0).any()


def test_powerlaw_full_size_matches_spec():
    """The 262,144-row configuration: nnz near the spec's ~1.23M."""
    p = D.gen_powerlaw(262144, seed=0)
    assert 1_150_000 < p.nnz < 1_300_000
    assert np.diff(p.rowPtr).max() <= 4096


def test_autotune_cache_file_on_host(tmp_path):
    """A cache file drives DASPMM_ALG_AUTO without any device work."""
    L = D.lib()
    L.daspmm_tune_clear()
    p = tmp_path / "tune.txt"
    # layout nv dtype nr nnz p50 p90 p99 max us | alg vec L S cf chunk snap block pipe
    p.write_text("# daspmm autotune cache v1\n"
                 "0 128 0 5000 60000 7 31 127 900 12.500 1 4 8 4 1 0 0 256 1\n")
    assert L.daspmm_tune_load(str(p).encode()) == 0
    c = D.default_config(D.Alg.AUTO, 0, 5000, 5000, 60000, 128)
    assert (c.alg, c.vec, c.lanes_col, c.lanes_nnz) == (1, 4, 8, 4)
    c2 = D.default_config(D.Alg.AUTO, 0, 5001, 5001, 60000, 128)   # untuned: rule of thumb
    assert c2.alg == 4
    out = tmp_path / "out.txt"
    assert L.daspmm_tune_save(str(out).encode()) == 0
    assert "0 128 0 5000 60000" in out.read_text()
    L.daspmm_tune_clear()
