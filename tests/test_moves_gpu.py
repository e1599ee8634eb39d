"""The reference's richer move set on the GPU annealer: step adaptation with
the cooling cycle (SQS_JOB_ADAPT), collective set moves (SQS_JOB_COLLECTIVE),
kicks of overlapped replicas (SQS_JOB_KICK), the quench of every replica
at exchange rounds (SQS_JOB_QUENCH_ALL) and the certificate of every replica
at checkpoints (SQS_JOB_CERT_ALL).  Each option runs to a
certified packing, changes the trajectory, and keeps a job's result
independent of batching, slicing and launch shape."""
from __future__ import annotations

import math
from dataclasses import replace

import pytest

pytestmark = pytest.mark.gpu

KEYS = ("L", "L_cert", "L_polished", "proposals", "accepted", "shrinks", "improvements",
        "exchange_attempts", "exchange_accepts", "q")
OPTIONS = [dict(adapt=True), dict(collective=True), dict(kick=True), dict(quench_all=True),
           dict(adapt=True, collective=True, kick=True, quench_all=True)]


def _job(n=40, seed=13, sweeps=200, replicas=16, **kw):
    from sqs.anneal import AnnealJob, jittered_grid
    xya, L0 = jittered_grid(n, seed=seed)
    args = dict(L0=L0, replicas=replicas, sweeps=sweeps, exchange_every=10, tmin=1e-4, tmax=5e-2, seed=seed,
                polish_iters=50)
    args.update(kw)
    return AnnealJob(xya, **args)


@pytest.mark.parametrize("opts", OPTIONS, ids=lambda o: "+".join(o))
def test_move_options_are_reproducible(ctx, oracle, opts):
    from sqs.anneal import anneal_batch
    job = _job(**opts)
    plain = anneal_batch([_job()], ctx=ctx)[0]
    alone = anneal_batch([job], ctx=ctx)[0]
    assert alone["status"] == 0, alone["reason"]
    assert alone["proposals"] == 16 * 200 * 40
    assert alone["launch"]["overflows"] == 0
    assert alone["q"] != plain["q"] or alone["accepted"] != plain["accepted"]  # the option acts
    assert alone["certified"], alone["reason"]
    ok, L, reason, _ = oracle.certify(40, alone["rows"])
    assert ok and L == alone["L"], reason
    mixed = anneal_batch([_job(n=25, seed=2), job, _job(n=60, seed=5, **opts)], ctx=ctx)[1]
    sliced = anneal_batch([job], ctx=ctx, slice_sweeps=50)[0]
    wide = anneal_batch([replace(job, cluster=4)], ctx=ctx)[0]
    for k in KEYS:
        assert mixed[k] == alone[k], ("mixed", k)
        assert sliced[k] == alone[k], ("sliced", k)
        assert wide[k] == alone[k], ("cluster 4", k)


@pytest.mark.parametrize("opts", [dict(cert_all=True), dict(cert_all=True, adapt=True, collective=True, kick=True),
                                  dict(quench_steps=8), dict(quench_all=True, quench_steps=4, kick=True)],
                         ids=lambda o: "+".join(f"{k}={v}" for k, v in o.items()))
def test_checkpoint_options_are_reproducible(ctx, oracle, opts):
    """SQS_JOB_CERT_ALL measures every replica's dilation-certified side at
    each checkpoint, whatever its overlap energy; SQS_JOB_QUENCH_STEPS(k)
    gives the checkpoint quench 16 k iterations with no slow-progress exit.
    Either way the job runs to a result the oracle certifies, and that result
    does not depend on batching, slicing or launch shape."""
    from sqs.anneal import anneal_batch
    job = _job(**opts)
    alone = anneal_batch([job], ctx=ctx)[0]
    assert alone["status"] == 0, alone["reason"]
    assert alone["proposals"] == 16 * 200 * 40
    assert alone["launch"]["overflows"] == 0
    if opts.get("cert_all"):
        assert alone["improvements"] >= 1
    assert alone["certified"], alone["reason"]
    ok, L, reason, _ = oracle.certify(40, alone["rows"])
    assert ok and L == alone["L"], reason
    mixed = anneal_batch([_job(n=25, seed=2), job, _job(n=60, seed=5, **opts)], ctx=ctx)[1]
    sliced = anneal_batch([job], ctx=ctx, slice_sweeps=50)[0]
    wide = anneal_batch([replace(job, cluster=4)], ctx=ctx)[0]
    for k in KEYS:
        assert mixed[k] == alone[k], ("mixed", k)
        assert sliced[k] == alone[k], ("sliced", k)
        assert wide[k] == alone[k], ("cluster 4", k)


def test_adaptation_steers_acceptance(ctx):
    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid
    # an exact 6 x 6 grid at side 6: every square touches its neighbours, so
    # large fixed steps at low temperature are almost always rejected; the
    # adapted steps shrink (down to the factor's floor of 0.1 on the coldest
    # rungs) and are accepted many times more often
    xya, _ = jittered_grid(36, jitter=0.0, angle_hi=1e-9, seed=1)
    args = dict(L0=6.0, replicas=8, sweeps=300, exchange_every=10, tmin=1e-6, tmax=1e-4, sigma_xy=0.1,
                sigma_a=0.3, seed=4, polish_iters=0)
    fixed = anneal_batch([AnnealJob(xya, **args)], ctx=ctx)[0]
    adapt = anneal_batch([AnnealJob(xya, adapt=True, **args)], ctx=ctx)[0]
    rf = fixed["accepted"] / fixed["proposals"]
    ra = adapt["accepted"] / adapt["proposals"]
    assert ra > 10 * rf and 0.005 < ra < 0.6, (rf, ra)


def test_replicas_start_from_a_portfolio(ctx):
    """Per-replica starts (sqs_job.xya_rep) from the structured portfolio: the
    job's result is the same alone, sliced and served, and differs from
    starting every replica at the seed."""
    from sqs.anneal import anneal_batch, portfolio
    from sqs.serve import Server
    base = _job(n=30, seed=21, sweeps=150, replicas=8)
    starts = portfolio(base.xya, base.L0, 8, seed=3)
    job = replace(base, xya_rep=starts)
    alone = anneal_batch([job], ctx=ctx)[0]
    plain = anneal_batch([base], ctx=ctx)[0]
    assert alone["status"] == 0
    assert alone["q"] != plain["q"] or alone["accepted"] != plain["accepted"]
    sliced = anneal_batch([job], ctx=ctx, slice_sweeps=30)[0]
    with Server(ctx, hbm_bytes=64 << 20, max_active=2, slice_sweeps=30) as srv:
        jid = srv.submit(job)
        for _ in range(100):
            if srv.step() == 0:
                break
        served = srv.poll(jid)
    for k in KEYS:
        assert sliced[k] == alone[k], ("sliced", k)
        assert served[k] == alone[k], ("served", k)


def test_proposal_counted_budgets_equal_sweep_counted_ones(ctx):
    """A budget of -k n proposals and checkpoints every -n proposals are the
    same job as k sweeps with a checkpoint every sweep, bit for bit; a
    checkpoint between sweeps (every 7 proposals) runs and differs."""
    from sqs.anneal import anneal_batch
    n = 30
    a = _job(n=n, sweeps=60, exchange_every=1, replicas=8)
    b = replace(a, sweeps=-60 * n, exchange_every=-n)
    c = replace(a, sweeps=-60 * n, exchange_every=-7)
    ra, rb, rc = anneal_batch([a, b, c], ctx=ctx)
    for k in KEYS:
        assert ra[k] == rb[k], k
    assert ra["sweeps"] == rb["sweeps"] == 60
    assert rc["status"] == 0 and rc["proposals"] == 8 * 60 * n
    assert rc["exchange_attempts"] > 4 * ra["exchange_attempts"]


def _target_job(**kw):
    # a 7-column grid of 48 squares in a side-7.5 box: certified sides below
    # the initial side exist, so the ladders improve on it
    args = dict(n=48, L0=7.5, sweeps=-48 * 60, exchange_every=-24, replicas=16, tmin=1e-11, tmax=1e-4,
                shrink=0.001 / 7,
                polish_iters=100, targets=True, ladders=2, adapt=True, kick=True, quench_all=True, cert_all=True,
                quench_steps=4)
    args.update(kw)
    return _job(**args)


def test_target_ladders_follow_the_reference_offsets(ctx, oracle):
    """Under SQS_JOB_TARGETS every rung anneals in side max(sqrt n, B (1 -
    shrink m)) below the best side B with the reference's offsets m; ladders
    repeat the temperatures of their rungs; the job certifies a packing."""
    from sqs.anneal import anneal_batch
    job = _target_job()
    r = anneal_batch([job], ctx=ctx, trace=True)[0]
    assert r["status"] == 0, r["reason"]
    assert r["certified"], r["reason"]
    ok, L, reason, _ = oracle.certify(job.n, r["rows"])
    assert ok and L == r["L"], reason
    t = r["trace"]
    mults = [0.02, 0.1, 0.4, 1.0, 2.5, 5.0, 10.0, 20.0]
    B = max(t["side"]) / (1 - job.shrink * 0.02)
    for rep in range(job.replicas):
        k = int(t["rung"][rep])
        want = max(math.sqrt(job.n) + 1e-6, B * (1 - job.shrink * mults[k % 8]))
        assert t["side"][rep] == pytest.approx(want, rel=1e-5)
    temp = {int(k): float(T) for k, T in zip(t["rung"], t["temperature"])}
    for k in range(8):
        assert temp[k] == temp[k + 8]
    assert r["improvements"] >= 1
    assert B <= job.L0 + 1e-6


def test_target_ladders_are_reproducible(ctx):
    from sqs.anneal import anneal_batch
    job = _target_job()
    alone = anneal_batch([job], ctx=ctx)[0]
    mixed = anneal_batch([_job(n=25, seed=2), job, _target_job(n=60, seed=5)], ctx=ctx)[1]
    sliced = anneal_batch([job], ctx=ctx, slice_sweeps=7)[0]
    wide = anneal_batch([replace(job, cluster=4)], ctx=ctx)[0]
    for k in KEYS:
        assert mixed[k] == alone[k], ("mixed", k)
        assert sliced[k] == alone[k], ("sliced", k)
        assert wide[k] == alone[k], ("cluster 4", k)


def test_group_quench_is_width_independent(ctx):
    """Under SQS_JOB_QUENCH_ALL every replica is quenched at once by a group
    of warps whose size the launch picks from how many clusters must stay
    resident: up to four warps a replica for one job alone, fewer when 120
    copies share the launch.  The quench's sums are integers, so every copy
    ends exactly where the job alone does."""
    from sqs.anneal import anneal_batch
    job = _job(replicas=16, cluster=4, adapt=True, kick=True, quench_all=True, quench_steps=4, cert_all=True)
    alone = anneal_batch([job], ctx=ctx)[0]
    assert alone["status"] == 0, alone["reason"]
    crowd = anneal_batch([job] * 120, ctx=ctx)
    assert all(r["status"] == 0 for r in crowd)
    for r in (crowd[0], crowd[57], crowd[-1]):
        for k in KEYS:
            assert r[k] == alone[k], k
