"""Launch shapes of the batched annealer: pinned cluster sizes and cell sides
leave a job's trajectory unchanged, the autotuner picks one of them (and an
exchange interval when asked), caches its choice per job class, and a sliced
run replays its slice loop as a CUDA graph with the unsliced result."""
from __future__ import annotations

from dataclasses import replace

import pytest

pytestmark = pytest.mark.gpu

KEYS = ("L", "L_cert", "L_polished", "proposals", "accepted", "shrinks", "improvements",
        "exchange_attempts", "exchange_accepts", "q")
CELLS = (1.59, 1.75, 1.95, 2.2)


def _job(n, seed, sweeps, replicas=16, **kw):
    from sqs.anneal import AnnealJob, jittered_grid
    xya, L0 = jittered_grid(n, seed=seed)
    args = dict(L0=L0, replicas=replicas, sweeps=sweeps, exchange_every=10, tmin=1e-3, tmax=1e-1, seed=seed,
                polish_iters=20)
    args.update(kw)
    return AnnealJob(xya, **args)


def test_pinned_shapes_give_the_same_trajectory(ctx):
    from sqs.anneal import anneal_batch
    base = _job(48, 11, 200)
    ref = anneal_batch([base], ctx=ctx)[0]
    assert ref["launch"]["cluster_ctas"] == 1 and ref["launch"]["overflows"] == 0
    for cs in (1, 2, 4, 8):
        for k, cell in enumerate(CELLS):
            r = anneal_batch([replace(base, cluster=cs, cell_index=k)], ctx=ctx)[0]
            assert r["launch"]["cluster_ctas"] == cs and r["launch"]["replicas_per_cta"] == 16 // cs
            assert abs(r["launch"]["cell_side"] - cell) < 1e-6
            assert r["launch"]["overflows"] == 0
            for key in KEYS:
                assert r[key] == ref[key], (cs, k, key)


def test_autotuner_choice_is_cached_and_result_unchanged(ctx):
    from sqs.anneal import anneal_batch, autotune
    job = _job(60, 2, 100, autotune=True)
    t1 = autotune(job, ctx=ctx)
    assert t1["trials"] > 0 and t1["us_per_sweep"] > 0
    assert t1["cluster_ctas"] * t1["replicas_per_cta"] == 16
    assert any(abs(t1["cell_side"] - c) < 1e-6 for c in CELLS)
    assert t1["exchange_every"] == 10
    t2 = autotune(job, ctx=ctx)
    assert t2["trials"] == 0
    assert (t2["cluster_ctas"], t2["cell_side"]) == (t1["cluster_ctas"], t1["cell_side"])
    other = _job(20, 4, 100)
    tuned = anneal_batch([job, other], ctx=ctx)
    plain = anneal_batch([replace(job, autotune=False), other], ctx=ctx)
    assert tuned[0]["launch"]["cluster_ctas"] == t1["cluster_ctas"]
    assert tuned[0]["launch"]["overflows"] == 0 and plain[0]["launch"]["overflows"] == 0
    for a, b in zip(tuned, plain):
        for key in KEYS:
            assert a[key] == b[key], key


def test_autotuned_exchange_interval(ctx):
    from sqs import SQSError
    from sqs.anneal import anneal_batch, autotune
    job = _job(24, 6, 200, exchange_every=0, autotune=True)
    t = autotune(job, ctx=ctx)
    assert t["exchange_every"] in (1, 2, 5, 10, 20, 50, 100)
    r = anneal_batch([job], ctx=ctx)[0]
    assert r["status"] == 0 and r["launch"]["exchange_every"] == t["exchange_every"]
    with pytest.raises(SQSError):  # 0 needs the autotuner
        anneal_batch([replace(job, autotune=False)], ctx=ctx)
    with pytest.raises(SQSError):  # a pinned shape excludes the tuner
        anneal_batch([replace(job, exchange_every=10, cluster=2)], ctx=ctx)
    with pytest.raises(SQSError):  # 3 does not divide 16 replicas
        anneal_batch([replace(job, exchange_every=10, autotune=False, cluster=3)], ctx=ctx)


def test_sliced_run_replays_a_graph(ctx):
    from sqs.anneal import anneal_batch
    a = _job(12, 7, 600, replicas=8)
    whole = anneal_batch([a], ctx=ctx)[0]
    before = ctx.graph_replays()
    sliced = anneal_batch([a], ctx=ctx, slice_sweeps=50)[0]
    assert ctx.graph_replays() - before == 12
    for key in KEYS:
        assert sliced[key] == whole[key], key
