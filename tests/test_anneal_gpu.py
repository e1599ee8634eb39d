"""Anneal-and-certify jobs on the GPU: the returned packings pass the
certifier (and the oracle restatement of the reference certifier), results
do not depend on batching or slicing, clusters of CTAs serve large jobs."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("L", "L_cert", "L_polished", "proposals", "accepted", "shrinks", "improvements",
        "exchange_attempts", "exchange_accepts", "q")


def plain_job(n=10, seed=42, sweeps=2000, **kw):
    from sqs.anneal import AnnealJob, jittered_grid
    xya, L0 = jittered_grid(n, seed=seed)
    args = dict(L0=L0, replicas=8, sweeps=sweeps, exchange_every=10, tmin=1e-3, tmax=1e-1, seed=seed)
    args.update(kw)
    return AnnealJob(xya, **args)


def test_plain_job_is_certified(ctx, oracle):
    from sqs.anneal import anneal_batch
    r = anneal_batch([plain_job()], ctx=ctx)[0]
    assert r["status"] == 0 and r["certified"], r["reason"]
    # a dilation-certified side within 0.1% of the 4x4 grid start (the
    # 20,000-sweep run of the same job leaves the grid topology for ~3.71)
    assert math.sqrt(10) <= float(r["L"]) < 4.004
    assert r["proposals"] == 8 * 2000 * 10
    assert r["shrinks"] >= 1 and r["exchange_attempts"] > 0
    ok, L, reason, _ = oracle.certify(10, r["rows"])
    assert ok and L == r["L"], reason
    # the certified side is at most the FP64 recompute's side times the dilation
    assert float(r["L"]) <= r["L_polished"] * r["dilation"] * (1 + 1e-12)


def test_same_result_alone_in_a_mix_and_sliced(ctx):
    from sqs.anneal import anneal_batch
    a = plain_job(n=12, seed=7, sweeps=600)
    others = [plain_job(n=30, seed=3, sweeps=300), plain_job(n=5, seed=9, sweeps=900, replicas=4)]
    alone = anneal_batch([a], ctx=ctx)[0]
    mixed = anneal_batch([others[0], a, others[1]], ctx=ctx)[1]
    sliced = anneal_batch([a], ctx=ctx, slice_sweeps=70)[0]
    for k in KEYS:
        assert alone[k] == mixed[k], k
        assert alone[k] == sliced[k], k


def test_cluster_of_ctas_for_a_large_ladder(ctx, oracle):
    from sqs.anneal import anneal_batch
    # 300 squares x 32 replicas do not fit one SM's shared memory: two CTAs
    # of 16 replicas exchange over distributed shared memory.
    job = plain_job(n=300, seed=5, sweeps=40, replicas=32, polish_iters=400)
    r = anneal_batch([job], ctx=ctx)[0]
    assert r["status"] == 0, r["reason"]
    assert r["proposals"] == 32 * 40 * 300
    assert r["exchange_attempts"] > 0
    assert r["certified"], r["reason"]
    ok, L, reason, _ = oracle.certify(300, r["rows"])
    assert ok and L == r["L"], reason


def test_determinism_and_seed_dependence(ctx):
    from sqs.anneal import anneal_batch
    r1, r2, r3 = anneal_batch([plain_job(seed=11, sweeps=300), plain_job(seed=11, sweeps=300),
                               plain_job(seed=12, sweeps=300)], ctx=ctx)
    assert r1["q"] == r2["q"] and r1["accepted"] == r2["accepted"]
    assert r1["accepted"] != r3["accepted"]


def test_job_errors(ctx):
    from sqs import SQSError
    from sqs.anneal import AnnealJob, anneal_batch
    good = plain_job(sweeps=10)
    for bad in (dict(replicas=65), dict(L0=100.0), dict(sigma_xy=0.0), dict(shrink=0.5), dict(tmin=0.0)):
        job = plain_job(sweeps=10, **bad)
        with pytest.raises(SQSError):
            anneal_batch([good, job], ctx=ctx)
    nan = plain_job(sweeps=10)
    nan.xya[0, 0] = float("nan")
    with pytest.raises(SQSError):
        anneal_batch([nan], ctx=ctx)
    # 40 squares piled on one point overflow a cell: a job error, not a crash
    pile = AnnealJob(np.tile([[2.0, 2.0, 0.3]], (40, 1)), L0=8.0, replicas=2, sweeps=20, seed=1)
    r = anneal_batch([pile, good], ctx=ctx)
    assert r[0]["status"] < 0 and "cell capacity" in r[0]["reason"]
    assert r[1]["status"] == 0


def test_zero_sweeps_returns_input_unimproved(ctx):
    from sqs.anneal import anneal_batch
    r = anneal_batch([plain_job(sweeps=0)], ctx=ctx)[0]
    assert r["status"] == 0 and not r["certified"] and r["proposals"] == 0


def test_job_without_a_certified_state_is_rescued(ctx, oracle):
    """Two sweeps at a tiny temperature leave the jittered (overlapping) grid
    uncertified; the coldest replica's final state is then polished from
    scratch into a certified packing -- identically alone, in a batch and
    served -- while a job that asks for no polish returns none."""
    from dataclasses import replace

    from sqs.anneal import anneal_batch
    from sqs.serve import Server
    job = plain_job(n=30, seed=8, sweeps=2, replicas=8, exchange_every=1, tmin=1e-11, tmax=1e-10,
                    polish_iters=400)
    r = anneal_batch([job], ctx=ctx)[0]
    assert r["status"] == 0 and r["certified"], r["reason"]
    ok, L, reason, _ = oracle.certify(30, r["rows"])
    assert ok and L == r["L"], reason
    none = anneal_batch([replace(job, polish_iters=0)], ctx=ctx)[0]
    assert not none["certified"]
    mixed = anneal_batch([plain_job(n=12, seed=1, sweeps=50), job], ctx=ctx)[1]
    with Server(ctx, hbm_bytes=32 << 20, max_active=2, slice_sweeps=1) as srv:
        jid = srv.submit(job)
        while srv.step():
            pass
        served = srv.poll(jid)
    for k in KEYS:
        assert mixed[k] == r[k] and served[k] == r[k], k


def test_paired_proposals_equal_one_at_a_time(ctx):
    """Plain jobs evaluate two proposals at once (one per half-warp) and
    evaluate the second again when the first's accepted move touched what it
    read.  The trajectory must be the one-at-a-time trajectory (SQS_JOB_SERIAL)
    bit for bit, on grids from 4 x 4 cells up, alone and batched, in every
    launch shape."""
    from sqs.anneal import anneal_batch
    cases = [dict(n=20, replicas=8, sweeps=300), dict(n=60, replicas=16, sweeps=200),
             dict(n=200, replicas=32, sweeps=60), dict(n=500, replicas=16, sweeps=20),
             dict(n=976, replicas=16, sweeps=10), dict(n=130, replicas=64, sweeps=40, cluster=8)]
    jobs = [plain_job(seed=50 + k, polish_iters=20, **c) for k, c in enumerate(cases)]
    serial = [plain_job(seed=50 + k, polish_iters=20, serial=True, **c) for k, c in enumerate(cases)]
    batched = anneal_batch(jobs, ctx=ctx)
    alone_serial = [anneal_batch([j], ctx=ctx)[0] for j in serial]
    for k, (a, b) in enumerate(zip(batched, alone_serial)):
        assert a["accepted"] > 0, k
        for key in KEYS:
            assert a[key] == b[key], (cases[k], key)
    # another shape of the 200-square job, paired, still the same
    other = anneal_batch([plain_job(seed=52, polish_iters=20, cluster=4, **cases[2])], ctx=ctx)[0]
    for key in KEYS:
        assert other[key] == alone_serial[2][key], key
