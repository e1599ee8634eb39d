"""The annealer and the FP64 recompute against the FP64 oracle, not against
themselves.

* Every replica's final FP32 state comes back with the annealer's running
  energy (its exact fixed-point sum of pair and wall terms), the same energy
  recomputed from scratch, and the FP64 dilation-certified side measured by
  the device function the checkpoints use (sqs_anneal_batch_trace).  The
  running energy equals the recompute bit for bit (nothing drifts); it agrees
  with the oracle's FP64 total of the same state within 1e-5 relative, with
  the reference's own absolute floor of 1e-5 (its device test of the search
  energy, cuda/tests/globaltest.cu:49); and the certified side equals the
  oracle's restatement of device_certified_side (seeded.cu:175-226) to a few
  ulps (CUDA's double sin/cos against the host's).
* Temperatures and step scales follow the reference's ladder, cooling cycle
  and rung scaling (seeded.cu:493-494, 506).
* Acceptance of single-square moves and of replica exchanges matches the
  oracle's CPU parallel tempering (ptsa_oracle.c) at fixed temperatures on
  the same problem: the same Metropolis and exchange rules on the same
  energy model.
* The FP64 energy / gradient entry point matches the oracle's pair_cached
  and smooth gradient to 1e-12 and central differences to 1e-7, the
  reference's device test (cuda/tests/seeded_test.cu:5-31).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ENERGY_REL = 1e-5   # FP32 energies against the FP64 oracle (relative) ...
ENERGY_ABS = 1e-5   # ... with the absolute floor of globaltest.cu:49
SIDE_REL = 1e-13    # FP64 certified side, GPU against host (trig differs by ulps)


def plain_jobs():
    """The plain single-instance configuration: n = 10, L0 = 4, jittered grid
    from seed 42, 8 replicas on 1e-3 .. 1e-1, 20,000 sweeps."""
    from sqs.anneal import AnnealJob, jittered_grid
    xya, L0 = jittered_grid(10, seed=42)
    return [AnnealJob(xya, L0=L0, replicas=8, sweeps=20000, exchange_every=10, tmin=1e-3, tmax=1e-1,
                      seed=42, polish_iters=200)]


def batched_jobs(count=24, sweeps=300):
    """A sample of the batched configuration: n uniform in [20, 400], 32
    replicas on 1e-4 .. 5e-2, sigma 0.02 / 0.05, exchange every 10 sweeps."""
    from sqs.anneal import AnnealJob, jittered_grid
    rng = np.random.default_rng(42)
    jobs = []
    for k in range(count):
        n = int(rng.integers(20, 401))
        xya, L0 = jittered_grid(n, seed=100 + k)
        jobs.append(AnnealJob(xya, L0=L0, replicas=32, sweeps=sweeps, exchange_every=10, tmin=1e-4, tmax=5e-2,
                              sigma_xy=0.02, sigma_a=0.05, seed=1000 + k, polish_iters=0))
    return jobs


def served_jobs_sample(sweeps=60):
    """A sample of the served stream's jobs: n from 5 to 1000, 16 to 64
    replicas, the move-set options mixed in."""
    from sqs.anneal import AnnealJob, jittered_grid
    rng = np.random.default_rng(7)
    jobs = []
    for k, n in enumerate([5, 17, 64, 180, 420, 777, 1000]):
        R = [16, 32, 64][k % 3] if n < 700 else 16
        xya, L0 = jittered_grid(n, seed=300 + k)
        jobs.append(AnnealJob(xya, L0=L0, replicas=R, sweeps=sweeps, exchange_every=10, tmin=1e-4, tmax=5e-2,
                              seed=int(rng.integers(1 << 30)), polish_iters=0, adapt=k % 2 == 1,
                              collective=k % 3 == 1, kick=k % 2 == 0))
    return jobs


def energy_errors(results, oracle):
    """Per replica: (relative, absolute) error of the running FP32 energy
    against the FP64 oracle's total on the same state and side, after
    checking that it equals its from-scratch recompute exactly."""
    rel, ab = [], []
    for r in results:
        t = r["trace"]
        assert t["cells_ok"]
        np.testing.assert_array_equal(t["energy"], t["energy_full"])
        xya = t["xya"].astype(np.float64)
        side = t["side"].astype(np.float64)
        eo, _, _ = oracle.total_batch(xya, side, grad=False)
        d = np.abs(t["energy"] - eo)
        ab.extend(d.tolist())
        rel.extend((d / np.maximum(eo, 1e-300)).tolist())
        tol = np.maximum(ENERGY_REL * eo, ENERGY_ABS)
        bad = np.nonzero(d > tol)[0]
        assert bad.size == 0, [(int(i), float(t["energy"][i]), float(eo[i])) for i in bad[:5]]
    return np.array(rel), np.array(ab)


@pytest.mark.parametrize("config", ["plain_n10", "batched_sample", "served_sample"])
def test_annealer_energy_matches_fp64_oracle(ctx, oracle, config):
    from sqs.anneal import anneal_batch
    jobs = {"plain_n10": plain_jobs, "batched_sample": batched_jobs, "served_sample": served_jobs_sample}[config]()
    res = anneal_batch(jobs, ctx=ctx, trace=True)
    for r in res:
        assert r["status"] == 0, r["reason"]
    rel, ab = energy_errors(res, oracle)
    assert rel.size == sum(j.replicas for j in jobs)
    print(f"{config}: {rel.size} replicas, max rel err {rel.max():.3e}, max abs err {ab.max():.3e}")


def test_running_energy_survives_slicing_and_moves(ctx, oracle):
    """Sliced runs (state reloaded from HBM), collective moves, kicks and
    quenches all keep the running energy equal to the recompute."""
    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid
    xya, L0 = jittered_grid(48, seed=5)
    job = AnnealJob(xya, L0=L0, replicas=16, sweeps=120, exchange_every=5, tmin=1e-4, tmax=5e-2, seed=9,
                    polish_iters=0, adapt=True, collective=True, kick=True, quench_all=True, cert_all=True)
    res = anneal_batch([job], ctx=ctx, slice_sweeps=15, trace=True)
    energy_errors(res, oracle)


def test_certified_side_matches_oracle(ctx, oracle):
    """The device certified side on every final replica of the plain and a
    batched sample: the dilation everywhere (the plain job's final states sit
    in a side below its best, so most need more than 1.008 and are rejected
    by both), the side wherever the dilation is accepted."""
    from sqs.anneal import anneal_batch
    jobs = plain_jobs() + batched_jobs(count=12, sweeps=400)
    res = anneal_batch(jobs, ctx=ctx, trace=True)
    measured = exact = lams = 0
    for r in res:
        t = r["trace"]
        for k in range(len(t["L_cert"])):
            L, lam, _ = oracle.certified_side(t["xya"][k].astype(np.float64))
            assert lam == pytest.approx(t["dilation"][k], rel=SIDE_REL), (k, lam, t["dilation"][k])
            lams += 1
            if L >= 1e8:
                assert t["L_cert"][k] >= 1e8
                continue
            measured += 1
            exact += L == t["L_cert"][k]
            assert t["L_cert"][k] == pytest.approx(L, rel=SIDE_REL), (k, L, t["L_cert"][k])
    assert lams == sum(j.replicas for j in jobs)
    assert measured >= 8, "too few replicas certified to compare"
    print(f"{lams} dilations and {measured} certified sides compared, {exact} sides bit-identical")


def test_temperature_and_step_schedule(ctx):
    """Rung temperatures tmin (tmax / tmin)^(k / (R - 1)) times the cooling
    factor 0.002^((x mod 200) / 199) of exchange round x, and step scales
    adapt x (0.15 + 1.85 k / (R - 1)) x sqrt(cool) with adapt in [0.1, 4]."""
    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid
    xya, L0 = jittered_grid(12, seed=3)
    jobs = []
    for k, (sweeps, xe) in enumerate([(10, 1), (57, 1), (450, 2), (90, 10)]):
        jobs.append(AnnealJob(xya, L0=L0, replicas=8, sweeps=sweeps, exchange_every=xe, tmin=1e-6, tmax=1e-2,
                              seed=k, polish_iters=0, adapt=True))
    jobs.append(AnnealJob(xya, L0=L0, replicas=5, sweeps=30, exchange_every=3, tmin=2e-5, tmax=3e-3, seed=9,
                          polish_iters=0))
    res = anneal_batch(jobs, ctx=ctx, trace=True)
    for j, r in zip(jobs, res):
        t = r["trace"]
        x = t["exchange_rounds"]
        assert x == j.sweeps // j.exchange_every
        cool = 0.002 ** ((x % 200) / 199.0) if j.adapt else 1.0
        R = j.replicas
        for rep in range(R):
            k = int(t["rung"][rep])
            want = j.tmin * (j.tmax / j.tmin) ** (k / (R - 1)) * cool
            assert t["temperature"][rep] == pytest.approx(want, rel=2e-5)
            if j.adapt:
                a = t["step_scale"][rep] / ((0.15 + 1.85 * k / (R - 1)) * math.sqrt(cool))
                assert 0.1 * (1 - 1e-5) <= a <= 4.0 * (1 + 1e-5), a
            else:
                assert t["step_scale"][rep] == 1.0
        assert sorted(t["rung"].tolist()) == list(range(R))


def test_acceptance_matches_oracle_parallel_tempering(ctx, oracle):
    """16 squares in a side-4 box (the optimum: no certified side can shrink
    it, so the side stays fixed), 8 rungs at fixed temperatures: the GPU
    annealer and the oracle's FP64 CPU annealer run the same Markov chain,
    so their move and exchange acceptance rates agree to sampling error."""
    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid
    xya, _ = jittered_grid(16, jitter=0.0, angle_hi=0.0, seed=1)
    jobs = [AnnealJob(xya, L0=4.0, replicas=8, sweeps=1500, exchange_every=5, tmin=1e-3, tmax=1e-1, sigma_xy=0.05,
                      sigma_a=0.1, shrink=0.0, seed=s, polish_iters=0) for s in range(4)]
    gpu = anneal_batch(jobs, ctx=ctx)
    cpu, _ = oracle.ptsa_batch(jobs)
    assert all(r["shrinks"] == 0 and r["launch"]["overflows"] == 0 for r in gpu)
    assert all(c["shrinks"] == 0 for c in cpu)
    ga = sum(r["accepted"] for r in gpu) / sum(r["proposals"] for r in gpu)
    ca = sum(c["accepted"] for c in cpu) / sum(c["proposals"] for c in cpu)
    gx = sum(r["exchange_accepts"] for r in gpu) / sum(r["exchange_attempts"] for r in gpu)
    cx = sum(c["exchange_accepts"] for c in cpu) / sum(c["exchange_attempts"] for c in cpu)
    print(f"move acceptance gpu {ga:.4f} oracle {ca:.4f}; exchange gpu {gx:.4f} oracle {cx:.4f}")
    assert 0.05 < ca < 0.95
    assert abs(ga - ca) < 0.03, (ga, ca)
    assert abs(gx - cx) < 0.06, (gx, cx)


def test_fp64_pair_energy_and_gradient(ctx, oracle):
    """The reference's device check of its FP64 pair (seeded_test.cu:5-31):
    10,000 random pairs, centres and angles uniform in (-1, 1); energy equal
    to the oracle's within 1e-12, the analytic gradient within 1e-7 of
    central differences (h = 1e-7) of the same entry point's energies."""
    from sqs.sat import energy_fp64
    rng = np.random.default_rng(832)
    m = 10000
    p = rng.uniform(-1, 1, (m, 3))
    q = rng.uniform(-1, 1, (m, 3))
    shift = np.array([10.0, 10.0, 0.0])  # far from the walls of a side-100 box
    states = np.stack([p + shift, q + shift], axis=1)
    e, g = energy_fp64(states, 100.0, ctx=ctx)
    eo = np.array([oracle.pair(a, b) for a, b in zip(states[:, 0], states[:, 1])])
    assert np.max(np.abs(e - eo)) <= 1e-12
    go = np.array([oracle.pair_cached(a, b, smooth=True)[1] for a, b in zip(states[:, 0], states[:, 1])])
    gp = np.array([x[0] for x in g])
    assert np.max(np.abs(gp - go)) <= 1e-12
    h = 1e-7
    fd = np.zeros((m, 3))
    for k in range(3):
        up, dn = states.copy(), states.copy()
        up[:, 0, k] += h
        dn[:, 0, k] -= h
        fd[:, k] = (energy_fp64(up, 100.0, ctx=ctx, grad=False)[0] -
                    energy_fp64(dn, 100.0, ctx=ctx, grad=False)[0]) / (2 * h)
    # the smooth gradient drops the derivative of |cos| / |sin| within 1e-6 of zero
    c = np.cos(states[:, 0, 2] - states[:, 1, 2])
    s = np.sin(states[:, 0, 2] - states[:, 1, 2])
    keep = (np.abs(c) > 1e-6) & (np.abs(s) > 1e-6)
    assert keep.sum() > 9990
    err = np.max(np.abs(fd - gp)[keep])
    assert err <= 1e-7, err
    assert np.count_nonzero(e) > 1000  # the sample is not trivially separated


def test_fp64_total_energy_and_gradient(ctx, oracle):
    """Packings with walls and many pairs, n up to 1000: energy within 1e-12
    relative of the oracle's total, gradient (the polish's smooth variant)
    within 1e-12 of the oracle's per coordinate."""
    from sqs.sat import energy_fp64
    from sqs.workloads import sat_microbench
    states, sides = [], []
    for k, n in enumerate([1, 2, 7, 57, 200, 640, 1000]):
        x, L = sat_microbench(configs=1, n=n, seed=50 + k, density_side=1.02)
        x[0, :, 2] = np.random.default_rng(k).uniform(-3, 3, n)  # angles beyond [0, pi/2) too
        states.append(x[0])
        sides.append(L[0] * 0.97)
    e, g = energy_fp64(states, np.array(sides), ctx=ctx)
    for k, (x, L) in enumerate(zip(states, sides)):
        eo, go = oracle.total_smooth(x, L)
        assert e[k] == pytest.approx(eo, rel=1e-12, abs=1e-300)
        np.testing.assert_allclose(g[k], go, rtol=0, atol=1e-12 * max(1.0, np.abs(go).max()))


def test_fp64_energy_rejects_bad_input(ctx):
    from sqs import SQSError
    from sqs.sat import energy_fp64
    with pytest.raises(SQSError):
        energy_fp64([np.zeros((1001, 3))], 40.0, ctx=ctx)
    with pytest.raises(SQSError):
        energy_fp64([np.full((3, 3), np.nan)], 4.0, ctx=ctx)
    with pytest.raises(SQSError):
        energy_fp64([np.zeros((3, 3))], -1.0, ctx=ctx)
