"""Seeded synthetic workloads with the shapes of the reference's configurations.

* lowerstar_grid: Freudenthal lower-star filtration of a G^3 grid of smoothed
  Gaussian noise (the 64^3, sigma 2 single-matrix workload).
* batch_of_rips: independent Rips complexes of uneven size - point counts
  log-uniform in [n_min, n_max], half in [0,1]^2 (up to dim 2) and half in
  [0,1]^3 (up to dim 3), each truncated at the radius giving an expected mean
  degree drawn uniformly from [deg_min, deg_max]; per-instance seeds.
* serving_stream: Poisson arrivals of requests mixing Rips complexes and
  lower-star grids, for the serving loop.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import gen


def lowerstar_grid(grid: int = 64, sigma: float = 2.0, seed: int = 2):
    return gen.lowerstar(grid, sigma, seed)


def rips_instance(seed: int, n_min: int, n_max: int, deg_min: float, deg_max: float, space_dim: int):
    rng = np.random.default_rng(seed)
    n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    k = float(rng.uniform(deg_min, deg_max))
    r = gen.rips_radius_for_degree(n, space_dim, k)
    return gen.rips(n, space_dim, seed, r, 2 if space_dim == 2 else 3), {"npts": n, "degree": k, "radius": r,
                                                                          "space_dim": space_dim, "seed": seed}


def _parallel(fn, args, threads: int | None):
    # the generators run in C and release the interpreter lock
    from concurrent.futures import ThreadPoolExecutor

    threads = threads or min(32, os.cpu_count() or 1)
    if threads <= 1:
        return [fn(*a) for a in args]
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda a: fn(*a), args))


def batch_of_rips(count: int = 512, seed: int = 4, n_min: int = 200, n_max: int = 5000, deg_min: float = 8.0,
                  deg_max: float = 40.0, threads: int | None = None):
    """(matrices, descriptions); half 2-D, half 3-D."""
    out = _parallel(rips_instance, [(seed * 1_000_003 + i, n_min, n_max, deg_min, deg_max, 2 if i % 2 == 0 else 3)
                                    for i in range(count)], threads)
    return [m for m, _ in out], [d for _, d in out]


def serving_specs(count: int, rate_per_s: float, seed: int = 5):
    """Requests (arrival time s, kind, description) with Poisson arrivals.

    Mix: Rips complexes of 300-20,000 points (2-D/3-D, mean degree 8-40, up to
    dim 3) and lower-star grids of 16^3-96^3 (sigma 1-3 voxels).
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate_per_s))
        if rng.random() < 0.75:
            out.append((t, "rips", {"seed": seed * 7919 + i, "space_dim": int(rng.choice([2, 3]))}))
        else:
            out.append((t, "lowerstar", {"grid": int(rng.integers(16, 97)), "sigma": float(rng.uniform(1.0, 3.0)),
                                         "seed": seed * 31 + i}))
    return out


def _materialize(kind, d):
    if kind == "rips":
        m, full = rips_instance(d["seed"], 300, 20000, 8.0, 40.0, d["space_dim"])
        return m, full
    return gen.lowerstar(d["grid"], d["sigma"], d["seed"]), d


def serving_stream(count: int, rate_per_s: float, seed: int = 5, threads: int | None = None):
    """Requests (arrival time s, kind, matrix, description) of serving_specs, generated in parallel."""
    specs = serving_specs(count, rate_per_s, seed)
    mats = _parallel(_materialize, [(k, d) for _, k, d in specs], threads)
    return [(t, k, m, d) for (t, k, _), (m, d) in zip(specs, mats)]
