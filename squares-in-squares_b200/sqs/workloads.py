"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (there is no public dataset for this problem; the
inputs are generated, never read from disk).
"""
from __future__ import annotations

import math

import numpy as np


def sat_microbench(configs: int = 4096, n: int = 200, seed: int = 42, density_side: float = 1.05):
    """Independent configurations of n unit squares: centres uniform in
    [0, L]^2 with L = 1.05 sqrt(n), angles uniform in [0, pi/2).

    Returns (xya float64 (configs, n, 3), side float64 (configs,))."""
    rng = np.random.default_rng(seed)
    L = density_side * math.sqrt(n)
    xy = rng.uniform(0.0, L, (configs, n, 2))
    a = rng.uniform(0.0, math.pi / 2, (configs, n, 1))
    return np.concatenate([xy, a], axis=2), np.full(configs, L)


def grid_state(n: int, pitch: float = 1.0, jitter: float = 0.0, angle_hi: float = 0.0, seed: int = 42):
    """Half-integer grid centres (ceil(sqrt(n)) columns) with optional uniform
    jitter in [-jitter, jitter] and angles uniform in [0, angle_hi)."""
    rng = np.random.default_rng(seed)
    w = math.isqrt(n - 1) + 1
    i = np.arange(n)
    xy = np.stack([(i % w + 0.5) * pitch, (i // w + 0.5) * pitch], axis=1)
    if jitter:
        xy = xy + rng.uniform(-jitter, jitter, xy.shape)
    a = rng.uniform(0.0, angle_hi, n) if angle_hi else np.zeros(n)
    return np.concatenate([xy, a[:, None]], axis=1)
