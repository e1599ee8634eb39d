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


def _log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def tilted_lattice(n: int, gap: float, theta: float, origin=(0.7, 0.9)):
    """n squares, all at angle theta, on a lattice along the squares' own axes
    with pitch 1 + gap: every lattice neighbour pair has exactly `gap` of
    clearance along a shared axis (to float64 accuracy).  Returns (n, 3)."""
    w = math.isqrt(n - 1) + 1
    i = np.arange(n)
    a, b = (i % w).astype(np.float64), (i // w).astype(np.float64)
    c, s = math.cos(theta), math.sin(theta)
    p = 1.0 + gap
    ox = origin[0] + (w * s if s > 0 else 0.0) * p
    x = ox + p * (a * c - b * s)
    y = origin[1] + p * (a * s + b * c)
    return np.stack([x, y, np.full(n, theta)], axis=1)


def rows_of(q, fmt: str = ".17g"):
    return [dict(square_id=str(k), x=format(float(x), fmt), y=format(float(y), fmt), angle=format(float(a), fmt))
            for k, (x, y, a) in enumerate(q)]


def grid_rows(n: int):
    w = math.isqrt(n - 1) + 1
    return [dict(square_id=str(i), x=f"{i % w}.5", y=f"{i // w}.5", angle="0") for i in range(n)]


def certify_corpus(count: int = 10000, seed: int = 42, n_lo: int = 5, n_hi: int = 1000,
                   overlap_frac: float = 0.05):
    """The interval-certifier batch: n log-uniform in [n_lo, n_hi]; half exact
    half-integer grids (every edge touching exactly), half tilted lattices
    with a clearance log-uniform in [1e-12, 1e-6]; a fraction of each with one
    square pushed 1e-10 into its neighbour.  Returns [(n, rows)]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = _log_uniform_int(rng, n_lo, n_hi)
        inject = rng.uniform() < overlap_frac and n >= 2
        if k % 2 == 0:
            if inject:
                q = grid_state(n)
                q[1, 0] -= 1e-10
                rows = grid_rows(n)
                rows[1]["x"] = format(float(q[1, 0]), ".17g")
            else:
                rows = grid_rows(n)
        else:
            gap = 10 ** rng.uniform(-12, -6)
            theta = float(rng.uniform(0.05, 1.5))
            q = tilted_lattice(n, gap, theta)
            if inject:
                # move square 1 toward square 0 by gap + 1e-10 along their shared axis
                d = q[1, :2] - q[0, :2]
                q[1, :2] -= d / np.linalg.norm(d) * (gap + 1e-10)
            rows = rows_of(q)
        out.append((n, rows))
    return out
