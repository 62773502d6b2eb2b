"""Seeded synthetic stand-ins for the benchmark configurations.

No public dataset is named for this path; the reference reads SuiteSparse
files that are not available here.  These generators reproduce the stated
shapes and distributions with fixed seeds:

  config 1  uniform 4096 x 4096, exactly 16 distinct columns per row, N = 32 (and 1)
  config 2  power-law graph, 262,144 rows, out-degree p(k) ~ (k+0.16)^-2.1 on
            [1, 4096], preferential-attachment columns, N = 128
  config 3  config 2's matrix and a 1M-row uniform-random matrix (average
            degree 8), N in {32, 128, 512}, BF16 / E4M3 storage
  config 4  512 instances: rows log-uniform in [1k, 64k], average degree
            log-uniform in [2, 64] with power-law row lengths, N = 64
  config 5  a pool of 64 matrices (rows log-uniform in [1k, 262k], half
            uniform-random, half power-law) and a Poisson request stream
"""
from __future__ import annotations

import math

import numpy as np

from . import gen_dense, gen_powerlaw, gen_random, gen_uniform


def powerlaw_mean(dmax: int, alpha: float = 2.1, shift: float = 0.16, dmin: int = 1) -> float:
    k = np.arange(dmin, dmax + 1, dtype=np.float64)
    p = (k + shift) ** -alpha
    return float((k * p).sum() / p.sum())


def config1():
    return gen_uniform(4096, 4096, 16, seed=0)


def config2():
    return gen_powerlaw(262144, seed=0)


def powerlaw_with_mean(nr: int, mean_deg: float, seed: int, nc: int | None = None):
    """Power-law row lengths scaled to an average degree (columns by
    preferential attachment)."""
    nc = nr if nc is None else nc
    dmax = min(4096, nc)
    scale = mean_deg / powerlaw_mean(dmax)
    return gen_powerlaw(nr, dmax=dmax, seed=seed, mean_scale=scale, nc=nc)


def config4_shapes(n: int = 512, seed: int = 4):
    """(rows, average degree) of the batched configuration's instances."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(math.log(1000), math.log(65536), n)).astype(int)
    deg = np.exp(rng.uniform(math.log(2), math.log(64), n))
    return [(int(r), float(d)) for r, d in zip(rows, deg)]


def config4(n: int = 512):
    return [powerlaw_with_mean(r, d, seed=i) for i, (r, d) in enumerate(config4_shapes(n))]


def config5_pool(n: int = 64, seed: int = 5):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        rows = int(math.exp(rng.uniform(math.log(1000), math.log(262144))))
        if i % 2 == 0:
            out.append(gen_random(rows, rows, float(rng.uniform(2, 16)), seed=1000 + i))
        else:
            out.append(gen_powerlaw(rows, dmax=min(4096, rows), seed=1000 + i))
    return out


def poisson_arrivals(rate_per_s: float, n: int, seed: int = 0):
    """Arrival times (s) of n requests of a Poisson process."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))


def dense(nrows: int, nv: int, seed: int = 1):
    return gen_dense(nrows * nv, seed=seed)
