"""Structured initial portfolio (sqs_portfolio, host code) against the
reference's own build_portfolio (seeded.cu:233-425, and the `packing`
program's copy in packing.cu, both compiled in oracle/_ref):
every chain's layout bit for bit, for sizes where topology candidates exist
and where none do; the per-chain jitter keeps centres in the container and
leaves group 0 untouched."""
from __future__ import annotations

import math

import numpy as np
import pytest


def _seed(n, pitch=1.0):
    w = math.isqrt(n - 1) + 1
    i = np.arange(n)
    return np.stack([(i % w + 0.5) * pitch, (i // w + 0.5) * pitch, np.zeros(n)], 1), w * pitch


@pytest.mark.parametrize("n,chains", [(2, 16), (5, 64), (10, 96), (11, 64), (17, 128), (26, 64), (50, 256),
                                      (101, 64), (300, 32)])
def test_portfolio_matches_reference(oracle, n, chains):
    if not oracle.ref_available():
        pytest.skip("compiled reference absent (make -C oracle ref)")
    from sqs.anneal import portfolio
    seed, L = _seed(n, 1.02)
    mine = portfolio(seed, L, chains, jitter=False)
    ref = oracle.ref_portfolio(n, L, seed, chains)
    assert mine.shape == ref.shape == (chains, n, 3)
    assert np.array_equal(mine, ref)
    if n >= 5:  # some chains leave the seed (topologies or grids)
        assert not all(np.array_equal(mine[b], seed) for b in range(chains))
    if (oracle.HERE / "_ref" / "libref_packing.so").exists():  # the packing program builds the same
        assert np.array_equal(mine, oracle.ref_portfolio_packing(n, L, seed, chains))
    flat = portfolio(seed, L, chains, structured=False, jitter=False)
    assert np.array_equal(flat, np.broadcast_to(seed, flat.shape))
    assert np.array_equal(oracle.ref_portfolio(n, L, seed, chains, structured=0), flat)


def test_portfolio_jitter():
    from sqs.anneal import portfolio
    seed, L = _seed(40, 1.05)
    a = portfolio(seed, L, 64, seed=5)
    b = portfolio(seed, L, 64, seed=5)
    c = portfolio(seed, L, 64, seed=6)
    base = portfolio(seed, L, 64, jitter=False)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    for ch in range(64):
        if ch % 8 == 0:
            assert np.array_equal(a[ch], base[ch])
        else:
            # centres jitter by at most 0.03 and are clamped into [0.5, L - 0.5]
            # (topology candidates may be up to 0.15 wider than L)
            d = np.abs(a[ch, :, :2] - np.clip(base[ch, :, :2], 0.5, L - 0.5))
            assert 0 < d.max() <= 0.03 + 1e-12
    # jittered chains are clamped into the container (unjittered group-0 chains
    # keep the reference's layouts, whose topologies may reach past it)
    jit = np.array([ch % 8 != 0 for ch in range(64)])
    assert a[jit, :, :2].min() >= 0.5 and a[jit, :, :2].max() <= L - 0.5
    assert np.all(a[jit, :, 2] >= 0) and np.all(a[jit, :, 2] < math.pi / 2)
