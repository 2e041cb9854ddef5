"""Seeded synthetic workloads (the reference's ocean u/v dataset is not distributed).

Each generator is the Gaussian-windowed linear-flow field described in
``csrc/gen.cpp`` (4-sigma window, N(0, 0.01^2) noise, joint rescale to [-1, 1]).

================  ==========================================================
workload          definition
================  ==========================================================
``cfg0``          2D u,v 2400x3600, 200 flows, sigma 40, eb 0.1 (CPU-runnable case)
``cfg1``          2D u,v 8192x8192, 2000 flows, sigma 60, eb 0.01 and 0.1
``cfg2``          3D u,v,w 384^3, 500 flows, sigma 20, eb 0.05
``cfg3``          256 2D fields, sides U{128..4096} each, one flow per 40x40
                  cells, sigma 40, eb drawn from {0.01, 0.05, 0.1}
``cfg4``          learned-bound training: 64 fields 2048x2048 of the cfg0
                  generator; evaluation 8192x8192 at eb 0.1
================  ==========================================================

"The cfg0 generator" at another size keeps cfg0's flow density (one flow per
43 200 cells) and sigma 40.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, lib

NOISE = 0.01
CFG0_DENSITY = 200 / (2400 * 3600)


def field_2d(seed: int, r1: int, r2: int, n_flows: int, sigma: float, noise: float = NOISE):
    U = np.empty((r1, r2), np.float32)
    V = np.empty((r1, r2), np.float32)
    _check(lib().cpsz_b200_generate_field_2d(seed, r1, r2, n_flows, sigma, noise, U.ctypes.data, V.ctypes.data))
    return U, V


def field_3d(seed: int, r1: int, r2: int, r3: int, n_flows: int, sigma: float, noise: float = NOISE):
    out = [np.empty((r1, r2, r3), np.float32) for _ in range(3)]
    _check(lib().cpsz_b200_generate_field_3d(seed, r1, r2, r3, n_flows, sigma, noise, *[a.ctypes.data for a in out]))
    return tuple(out)


def cfg0_like(seed: int, r1: int, r2: int):
    """The cfg0 generator at size r1 x r2 (flow density of cfg0, sigma 40)."""
    return field_2d(seed, r1, r2, max(1, round(CFG0_DENSITY * r1 * r2)), 40.0)


def cfg0(seed: int = 0):
    return field_2d(seed, 2400, 3600, 200, 40.0)


def cfg1(seed: int = 1):
    return field_2d(seed, 8192, 8192, 2000, 60.0)


def cfg2(seed: int = 2, n: int = 384):
    return field_3d(seed, n, n, n, 500, 20.0)


def batch_layout(base_seed: int = 3, n_fields: int = 256, lo: int = 128, hi: int = 4096):
    r1 = np.empty(n_fields, np.uint64)
    r2 = np.empty(n_fields, np.uint64)
    seeds = np.empty(n_fields, np.uint64)
    ebs = np.empty(n_fields, np.float64)
    _check(lib().cpsz_b200_batch_layout(base_seed, n_fields, lo, hi, r1.ctypes.data, r2.ctypes.data,
                                        seeds.ctypes.data, ebs.ctypes.data))
    return [(int(a), int(b), int(s), float(e)) for a, b, s, e in zip(r1, r2, seeds, ebs)]


def cfg3_field(r1: int, r2: int, seed: int):
    """One batched field: one flow per 40x40 cells, sigma 40."""
    return field_2d(seed, r1, r2, max(1, (r1 * r2) // 1600), 40.0)
