"""Serving loop: continuous batching with admission by HBM footprint; every
job's result in the mix equals its result alone."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu
KEYS = ("L", "L_cert", "L_polished", "proposals", "accepted", "shrinks", "exchange_attempts", "q")


def _job(n, seed, sweeps, replicas=8, **kw):
    from sqs.anneal import AnnealJob, jittered_grid
    xya, L0 = jittered_grid(n, seed=seed)
    return AnnealJob(xya, L0=L0, replicas=replicas, sweeps=sweeps, exchange_every=10, seed=seed, **kw)


def test_served_results_equal_alone(ctx):
    from sqs.anneal import anneal_batch
    from sqs.serve import Server
    jobs = [_job(10, 1, 300), _job(37, 2, 120, replicas=16), _job(5, 3, 500, replicas=4), _job(64, 4, 90)]
    alone = [anneal_batch([j], ctx=ctx)[0] for j in jobs]
    with Server(ctx, hbm_bytes=64 << 20, max_active=3, slice_sweeps=30) as srv:
        ids = [srv.submit(j) for j in jobs[:2]]
        srv.step()                       # the first two are running ...
        ids += [srv.submit(j) for j in jobs[2:]]  # ... when the others arrive
        got = {}
        for _ in range(100000):
            if srv.step() == 0:
                break
        for k, jid in enumerate(ids):
            got[k] = srv.poll(jid)
    for k in range(len(jobs)):
        assert got[k] is not None
        for key in KEYS:
            assert got[k][key] == alone[k][key], (k, key)


def test_admission_by_hbm_footprint(ctx):
    from sqs.serve import Server
    jobs = [_job(100, s, 40) for s in range(4)]
    per_job = 8 * 100 * 16 + 2 * 100 * 16 + 100 * 24  # replicas + scratch + best, bytes
    budget = 1 << 20                                  # room for one job at a time only
    assert per_job < budget < 2 * per_job + 4096 or budget > per_job
    with Server(ctx, hbm_bytes=budget, max_active=8, slice_sweeps=20) as srv:
        ids = [srv.submit(j) for j in jobs]
        peak_active = 0
        while True:
            left = srv.step()
            _, active, used = srv.info()
            peak_active = max(peak_active, active)
            assert used <= budget
            if left == 0:
                break
        results = [srv.poll(i) for i in ids]
    assert all(r is not None and r["status"] == 0 for r in results)
    assert peak_active >= 1


def test_cancel_and_unknown_ids(ctx):
    from sqs import SQSError
    from sqs.serve import Server
    with Server(ctx, hbm_bytes=32 << 20, max_active=1, slice_sweeps=10) as srv:
        a = srv.submit(_job(20, 5, 200))
        b = srv.submit(_job(20, 6, 200))
        srv.step()                 # a runs, b waits for the only slot
        srv.cancel(b)
        srv.cancel(a)              # a stops when its slice in flight ends
        for _ in range(100000):
            if srv.step() == 0:
                break
        ra, rb = srv.poll(a), srv.poll(b)
        assert ra["reason"] == "cancelled" and rb["reason"] == "cancelled"
        with pytest.raises(SQSError):
            srv.poll(a)            # collected already
        with pytest.raises(SQSError):
            srv.cancel(12345)


def test_poisson_stream_reports_latency(ctx):
    from sqs.serve import Server, poisson_arrivals, run_stream
    jobs = [_job(n, 10 + k, 60) for k, n in enumerate((8, 12, 20, 9, 15, 30))]
    arr = poisson_arrivals(len(jobs), rate=200.0, seed=1)
    with Server(ctx, hbm_bytes=64 << 20, max_active=4, slice_sweeps=20) as srv:
        results, stats = run_stream(srv, jobs, arr, timeout=120)
    assert stats["jobs"] == len(jobs)
    assert 0 < stats["p50_s"] <= stats["p99_s"]
    assert all(r is not None for r in results)


def test_proposal_sliced_server_equals_alone(ctx):
    """Per-job slices of about 300 proposals per replica (small jobs run many
    sweeps per step, large ones few): every result equals the job alone."""
    from sqs.anneal import anneal_batch
    from sqs.serve import Server
    jobs = [_job(6, 11, 400, replicas=4), _job(90, 12, 60, replicas=16), _job(25, 13, 200)]
    alone = [anneal_batch([j], ctx=ctx)[0] for j in jobs]
    with Server(ctx, hbm_bytes=64 << 20, max_active=3, slice_proposals=300) as srv:
        ids = [srv.submit(j) for j in jobs]
        steps = 0
        while srv.step():
            steps += 1
        got = [srv.poll(i) for i in ids]
    assert steps >= 3
    for a, b in zip(alone, got):
        for key in KEYS:
            assert a[key] == b[key], key


def test_server_counters_and_retirement_thread(ctx):
    """Every admitted job is retired exactly once by the retirement thread;
    slices and host phase times are counted; jobs of several cluster shapes
    (separate cohorts) all come back equal to their results alone."""
    from sqs.anneal import anneal_batch
    from sqs.serve import Server, poisson_arrivals, run_stream
    jobs = [_job(n, 30 + k, 80, replicas=r) for k, (n, r) in
            enumerate([(12, 4), (40, 16), (90, 32), (25, 8), (150, 64), (8, 2), (60, 16), (33, 32)])]
    alone = [anneal_batch([j], ctx=ctx)[0] for j in jobs]
    arr = poisson_arrivals(len(jobs), rate=500.0, seed=4)
    with Server(ctx, hbm_bytes=64 << 20, max_active=8, slice_proposals=500) as srv:
        results, stats = run_stream(srv, jobs, arr, timeout=120)
        st = srv.stats()
    assert stats["jobs"] == len(jobs)
    assert st["admitted"] == st["retired"] == len(jobs)
    assert st["slices"] >= len(jobs) and st["steps"] >= 1
    assert min(st["admit_s"], st["launch_s"], st["retire_s"], st["wait_s"]) >= 0.0
    for a, b in zip(alone, results):
        for key in KEYS:
            assert a[key] == b[key], key


def test_destroy_with_work_in_flight(ctx):
    """Closing a server while slices run and jobs wait for retirement stops
    its retirement thread and drains its streams: no hang, no fault, and the
    context stays usable for the next server."""
    import time

    from sqs.serve import Server
    jobs = [_job(n, 40 + k, 400, replicas=r) for k, (n, r) in enumerate([(30, 8), (120, 16), (12, 4), (60, 32)])]
    t0 = time.perf_counter()
    srv = Server(ctx, hbm_bytes=64 << 20, max_active=4, slice_proposals=200)
    for j in jobs:
        srv.submit(j)
    for _ in range(3):
        srv.step()
    srv.close()
    assert time.perf_counter() - t0 < 60
    with Server(ctx, hbm_bytes=64 << 20, max_active=2, slice_sweeps=50) as again:
        jid = again.submit(_job(10, 50, 100))
        while again.step():
            pass
        assert again.poll(jid)["status"] == 0
