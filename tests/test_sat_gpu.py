"""CUDA FP32 cell-list SAT energy + gradient against the FP64 all-pairs oracle
(the reference's energy model, seeded.cu:41-162), through the C ABI."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Tolerances stated by the reference's own device tests and the build goal:
# FP32 energies within 1e-5 relative of the FP64 energy (absolute floor 1e-6
# for near-zero energies); gradients within 1e-4 absolute + 1e-4 relative.
E_REL = 1e-5
E_ABS = 1e-6
G_TOL = 1e-4


def _run(ctx, xya, side, threads=None):
    from sqs import sat, _native as N
    x32 = np.ascontiguousarray(xya, dtype=np.float32)
    s32 = np.ascontiguousarray(np.broadcast_to(np.asarray(side, np.float32), (x32.shape[0],)))
    if threads is None:
        return sat.energy(x32, s32, ctx=ctx, grad=True, count=True), x32, s32
    configs, n, _ = x32.shape
    d_x = ctx.alloc(x32.shape, np.float32).upload(x32)
    d_s = ctx.alloc((configs,), np.float32).upload(s32)
    d_e = ctx.alloc((configs,), np.float32)
    d_g = ctx.alloc(x32.shape, np.float32)
    d_c = ctx.alloc((configs,), np.uint32)
    sat.energy_device(ctx, configs, n, d_x, d_s, d_e, d_g, d_c, threads=threads)
    out = (d_e.download(), d_g.download(), d_c.download())
    for d in (d_x, d_s, d_e, d_g, d_c):
        d.free()
    return out, x32, s32


def _check(oracle, out, x32, s32, grad_quantile=1.0):
    e, g, c = out
    eo, go, co = oracle.total_batch(x32.astype(np.float64), s32.astype(np.float64))
    err = np.abs(e.astype(np.float64) - eo)
    assert np.all(err <= E_REL * np.abs(eo) + E_ABS), (err.max(), eo[np.argmax(err)])
    gerr = np.abs(g.astype(np.float64) - go) - G_TOL * (1 + np.abs(go))
    bad = np.mean(gerr > 0)
    assert bad <= 1 - grad_quantile, bad
    assert np.all(np.abs(c.astype(np.int64) - co) <= 1)
    assert abs(int(c.sum()) - int(co.sum())) <= max(1, int(1e-4 * co.sum()))
    return np.max(err / np.maximum(np.abs(eo), 1e-30))


def test_microbench_distribution_parity(ctx, oracle):
    from sqs.workloads import sat_microbench
    xya, side = sat_microbench(configs=192, n=200, seed=42)
    out, x32, s32 = _run(ctx, xya, side)
    rel = _check(oracle, out, x32, s32, grad_quantile=0.9999)
    assert rel < E_REL
    assert out[2].mean() > 400  # about 520 candidate pairs per configuration


@pytest.mark.parametrize("threads", [32, 64, 128, 256, -2, -4, -8])
def test_cta_widths_agree(ctx, oracle, threads):
    from sqs.workloads import sat_microbench
    xya, side = sat_microbench(configs=40, n=200, seed=3)
    out, x32, s32 = _run(ctx, xya, side, threads=threads)
    _check(oracle, out, x32, s32, grad_quantile=0.9999)


def test_aligned_ties_follow_reference_gradient(ctx, oracle):
    # Axis-aligned overlapping grids: every overlapping pair has tied axes;
    # the gradient must follow the reference's own-axis-first choice.  The
    # pitches are dyadic so FP32 differences are exact and the ties are real
    # ties in both precisions (with a pitch like 0.9, FP32 rounding of dx vs
    # dy decides between two axes 1e-8 apart, a genuine kink of the energy).
    from sqs.workloads import grid_state
    states = np.stack([grid_state(49, pitch=p) for p in (0.75, 0.875, 0.9375, 1.0)])
    out, x32, s32 = _run(ctx, states, 6.5)
    _check(oracle, out, x32, s32)


def test_edge_cases(ctx, oracle):
    rng = np.random.default_rng(9)
    cases = []
    cases.append((np.array([[[0.2, 0.3, 0.7]]]), 1.0))                      # n=1, wall only
    cases.append((np.array([[[0.5, 0.5, 0.0], [1.5, 0.5, 0.0]]]), 2.0))     # exact contact
    cases.append((np.array([[[0.5, 0.5, 0.0], [0.5, 0.5, 0.0]]]), 2.0))     # coincident
    cases.append((np.array([[[1.0, 1.0, 0.3], [1.9, 1.4, 1.2]]]), 3.0))     # rotated overlap
    out_of_box = np.concatenate([rng.uniform(-3, 12, (3, 60, 2)), rng.uniform(-9, 9, (3, 60, 1))], axis=2)
    cases.append((out_of_box, 8.0))                                          # squares outside [0, L]
    sparse = np.concatenate([rng.uniform(0, 60, (2, 50, 2)), rng.uniform(0, 2, (2, 50, 1))], axis=2)
    cases.append((sparse, 60.0))                                             # sparse, capped grid
    for xya, side in cases:
        out, x32, s32 = _run(ctx, xya, side)
        _check(oracle, out, x32, s32)


def test_max_n_and_limits(ctx, oracle):
    from sqs import SQSError, sat
    from sqs.workloads import sat_microbench
    xya, side = sat_microbench(configs=6, n=1024, seed=5)
    out, x32, s32 = _run(ctx, xya, side)
    _check(oracle, out, x32, s32, grad_quantile=0.9999)
    e, g, c = sat.energy(np.zeros((0, 5, 3), np.float32), 3.0, ctx=ctx, count=True)
    assert e.shape == (0,)
    with pytest.raises(SQSError):
        sat.energy(np.zeros((1, 1025, 3), np.float32), 40.0, ctx=ctx)


@pytest.mark.parametrize("n", [200, 700])
def test_energy_and_gradient_are_deterministic(ctx, n):
    # gradients are summed with integer atomics, so even their order is irrelevant
    from sqs.workloads import sat_microbench
    xya, side = sat_microbench(configs=64, n=n, seed=1)
    (e1, g1, c1), _, _ = _run(ctx, xya, side)
    (e2, g2, c2), _, _ = _run(ctx, xya, side)
    assert np.array_equal(e1, e2) and np.array_equal(c1, c2) and np.array_equal(g1, g2)


def test_host_call_in_overlapped_chunks_equals_device_call(ctx, oracle):
    """A host-pointer call of 1,500 configurations runs as chunks whose
    uploads, kernels and downloads overlap on several streams; every energy,
    gradient and candidate count equals the single device-pointer launch bit
    for bit (configurations are independent), and agrees with the oracle."""
    from sqs import _native as N
    from sqs.workloads import sat_microbench
    xya, side = sat_microbench(configs=1500, n=120, seed=11)
    x32 = np.ascontiguousarray(xya, dtype=np.float32)
    s32 = np.ascontiguousarray(np.broadcast_to(np.asarray(side, np.float32), (x32.shape[0],)))
    hin, hs = N.PinnedArray(x32.shape, np.float32), N.PinnedArray(s32.shape, np.float32)
    hin.array[...] = x32
    hs.array[...] = s32
    he, hg = N.PinnedArray(s32.shape, np.float32), N.PinnedArray(x32.shape, np.float32)
    hc = N.PinnedArray(s32.shape, np.uint32)
    for _ in range(2):  # twice: the second call reuses the context's buffers
        N.check(N.lib().sqs_sat_energy_host(ctx.handle, x32.shape[0], x32.shape[1], N.ptr(hin.array, N._fp),
                                            N.ptr(hs.array, N._fp), N.ptr(he.array, N._fp), N.ptr(hg.array, N._fp),
                                            N.ptr(hc.array, N._u32p)))
        (e, g, c), _, _ = _run(ctx, x32, s32, threads=-4)
        assert np.array_equal(he.array, e) and np.array_equal(hg.array, g) and np.array_equal(hc.array, c)
    eo, _, _ = oracle.total_batch(x32[:100].astype(np.float64), s32[:100].astype(np.float64))
    assert np.all(np.abs(he.array[:100].astype(np.float64) - eo) <= E_REL * np.abs(eo) + E_ABS)
    for h in (hin, hs, he, hg, hc):
        h.free()


def test_reference_selftest_fixture(ctx, oracle):
    """The reference's device self-test (cuda/tests/selftest.cu:34-53) as a
    fixture: 100 configurations of 50 squares, centres U(-0.2, 12.2), angles
    U(-3.14, 3.14), plus axis-aligned pairs that touch exactly, or are 1e-6
    apart, across a cell boundary of the grid (side 12: 8 cells of 1.5).
    Energies within the stated tolerance of the FP64 oracle; the touching
    and separated pairs add no pair energy."""
    rng = np.random.default_rng(923)
    xya = np.concatenate([rng.uniform(-0.2, 12.2, (100, 50, 2)), rng.uniform(-3.14, 3.14, (100, 50, 1))], axis=2)
    out, x32, s32 = _run(ctx, xya, 12.0)
    _check(oracle, out, x32, s32, grad_quantile=0.99)
    # boundary pairs, well inside the container (no wall term)
    pairs = []
    for gap in (0.0, 1e-6):
        for b in (3.0, 4.5, 6.0):  # cell boundaries x = 1.5 k
            pairs.append([[b - 0.5, 6.0, 0.0], [b + 0.5 + gap, 6.0, 0.0]])
            pairs.append([[6.0, b - 0.5, 0.0], [6.0, b + 0.5 + gap, 0.0]])
    out, x32, s32 = _run(ctx, np.array(pairs, np.float64), 12.0)
    _check(oracle, out, x32, s32)
    assert np.all(out[0] == 0.0), out[0]


def test_reference_near_contact_grid(ctx, oracle):
    """The reference's large-n check (cuda/tests/globaltest.cu:49): a square
    grid at pitch 1.000001 -- every neighbour pair 1e-6 from contact once the
    centres are rounded to FP32 -- in a container that just holds it, through
    both kernels (n = 1024, one CTA per configuration; n = 256, one warp)."""
    for k in (32, 16):
        c = 0.5 + 1.000001 * np.arange(k)
        gx, gy = np.meshgrid(c, c)
        xya = np.stack([gx.ravel(), gy.ravel(), np.zeros(k * k)], axis=1)[None]
        out, x32, s32 = _run(ctx, xya, 1.000001 * k + 1e-6)
        _check(oracle, out, x32, s32)
