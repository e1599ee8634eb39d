"""The annealer's checkpoint quench sums a pair list instead of scanning cell
lists while no centre has moved more than 0.085 per axis since the list was
built.  The list holds the pairs (i < j) of each square's 3 x 3 block of cells
(cells at least 1.59 wide, edge cells clamped) closer than sqrt(2.75); the
claim is that it then holds every pair within the energy cut-off
(d^2 < 2.000001), so the list's energy and gradient equal the full ones.
This checks that claim on the CPU, in FP32 as the kernel computes it, on
random, dense, out-of-box and boundary-hugging configurations."""
from __future__ import annotations

import numpy as np

CUT2 = np.float32(2.000001)
LIST_CUT2 = np.float32(2.75)
STEP = 0.085
CELL = 1.59


def _cells(x, L, G):
    inv = np.float32(G) / np.float32(L)
    c = np.floor(x.astype(np.float32) * inv).astype(np.int64)
    return np.clip(c, 0, G - 1)


def _pair_list(xy, L):
    G = max(1, int(np.float32(L) / np.float32(CELL)))
    cx, cy = _cells(xy[:, 0], L, G), _cells(xy[:, 1], L, G)
    n = len(xy)
    out = set()
    for i in range(n):
        near = np.nonzero((np.abs(cx - cx[i]) <= 1) & (np.abs(cy - cy[i]) <= 1))[0]
        for j in near[near > i]:
            ex = np.float32(xy[j, 0] - xy[i, 0])
            ey = np.float32(xy[j, 1] - xy[i, 1])
            if ex * ex + ey * ey < LIST_CUT2:
                out.add((i, int(j)))
    return out


def _within_cut(xy):
    n = len(xy)
    d = xy[None, :, :] - xy[:, None, :]
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(np.float32)
    i, j = np.nonzero(np.triu(d2 < CUT2, 1))
    return set(zip(i.tolist(), j.tolist()))


def _check(xy, L, rng, moves=6):
    xy = xy.astype(np.float32)
    plist = _pair_list(xy, L)
    for _ in range(moves):
        step = rng.uniform(-STEP, STEP, xy.shape).astype(np.float32)
        # push some squares to the bound exactly
        edge = rng.random(xy.shape) < 0.3
        step[edge] = np.float32(STEP) * np.sign(step[edge])
        moved = (xy + step).astype(np.float32)
        missing = _within_cut(moved) - plist
        assert not missing, sorted(missing)[:5]


def test_random_and_dense_configurations():
    rng = np.random.default_rng(5)
    for n, density in [(40, 0.6), (120, 1.0), (200, 1.3), (300, 1.8)]:
        L = float(np.sqrt(n / density))
        xy = rng.uniform(0.0, L, (n, 2))
        _check(xy, L, rng)


def test_squares_outside_the_box_and_on_cell_edges():
    rng = np.random.default_rng(9)
    L = 9.0
    G = int(L / CELL)
    w = L / G
    # centres on cell boundaries, and pairs 1.5842 apart per axis (the bound)
    pts = []
    for k in range(G):
        for m in range(G):
            pts.append((k * w + 1e-6, m * w - 1e-6))
    pts += [(1.0, 1.0), (1.0 + 1.5842, 1.0), (1.0, 1.0 + 1.5842), (1.0 + 1.17, 1.0 + 1.17)]
    pts += [(-2.0, 3.0), (L + 1.5, -0.7), (L + 0.2, L + 0.4)]  # clamped into edge cells
    xy = np.array(pts, dtype=np.float64)
    _check(xy, L, rng, moves=20)


def test_many_seeds_small_boxes():
    rng = np.random.default_rng(13)
    for _ in range(30):
        n = int(rng.integers(5, 60))
        L = float(rng.uniform(2.5, 9.0))
        xy = rng.uniform(-0.3, L + 0.3, (n, 2))
        _check(xy, L, rng, moves=3)
