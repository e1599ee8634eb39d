"""The CPU oracle against the reference's golden vectors and, where it was
compiled here, against the reference's own code (oracle/_ref)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_pair_energy_matches_reference_golden(oracle):
    recs = json.loads((GOLDEN / "sat_pairs.json").read_text())
    for r in recs:
        e, g = oracle.pair(r["p"], r["q"], grad=True)
        assert e == r["e"]
        assert g.tolist() == r["g"]
        gb = np.zeros(3)
        p = np.ascontiguousarray(r["p"], dtype=np.float64)
        b = oracle.lib().sqo_boundary(p.ctypes.data_as(oracle._dp), r["wall_L"], gb.ctypes.data_as(oracle._dp))
        assert b == r["wall"]
        assert gb.tolist() == r["wall_g"]


def test_pair_gradient_matches_finite_differences(oracle):
    # Mirrors the reference's device test: 1e-7 against central differences
    # with h = 1e-7 on random pairs (cuda/tests/seeded_test.cu:65-80).
    rng = np.random.default_rng(832)
    worst = 0.0
    for _ in range(3000):
        p, q = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)
        _, g = oracle.pair(p, q, grad=True)
        for k in range(3):
            a, b = p.copy(), p.copy()
            a[k] += 1e-7
            b[k] -= 1e-7
            fd = (oracle.pair(a, q) - oracle.pair(b, q)) / 2e-7
            worst = max(worst, abs(fd - g[k]))
    assert worst < 1e-7


def test_certifier_cases_match_golden(oracle):
    cases = json.loads((GOLDEN / "certify_cases.json").read_text())
    assert len(cases) >= 50
    for c in cases:
        ok, L, reason, score = oracle.certify(c["n"], c["rows"])
        assert ok == c["ok"], c["name"]
        assert L == c["L"], c["name"]
        assert reason == c["reason"], c["name"]
        assert score == c["score"], c["name"]


def test_roundtrip_emulation(oracle):
    assert oracle.roundtrip("0.5") == "0.5"
    assert oracle.roundtrip("3") == "3.0"
    assert oracle.roundtrip("1.100000000000000010000000000001") == "1.1"
    assert oracle.roundtrip("0.10000000000000001") == "0.1"


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
def test_total_energy_bit_exact_vs_reference(oracle):
    rng = np.random.default_rng(7)
    for n, L in ((2, 1.5), (10, 4.0), (200, 1.05 * math.sqrt(200)), (57, 6.0)):
        xya = np.concatenate([rng.uniform(-0.5, L + 0.5, (6, n, 2)), rng.uniform(-3, 3, (6, n, 1))], axis=2)
        e, g, _ = oracle.total_batch(xya, L, threads=2)
        er, gr, _ = oracle.ref_total_batch(xya, L, threads=2)
        assert np.array_equal(e, er)
        assert np.array_equal(g, gr)


def _random_packing(rng, n, kind):
    if kind == "grid":
        w = math.isqrt(n - 1) + 1
        return [dict(square_id=str(i), x=f"{i % w}.5", y=f"{i // w}.5", angle="0") for i in range(n)]
    L = 1.3 * math.sqrt(n) + 1
    q = np.concatenate([rng.uniform(0, L, (n, 2)), rng.uniform(-7, 7, (n, 1))], axis=1)
    rows = [dict(square_id=str(i), x=repr(float(x)), y=repr(float(y)), angle=repr(float(a)))
            for i, (x, y, a) in enumerate(q)]
    if kind == "shuffled":
        rng.shuffle(rows)
    return rows


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
def test_certifier_bit_exact_vs_reference_random(oracle):
    rng = np.random.default_rng(11)
    seen = set()
    for trial in range(120):
        n = int(rng.integers(1, 40))
        kind = ("grid", "random", "shuffled")[trial % 3]
        rows = _random_packing(rng, n, kind)
        a = oracle.certify(n, rows)
        b = oracle.certify(n, rows, "ref")
        assert a[:3] == b[:3], (trial, a, b)
        assert a[3] == b[3]
        seen.add(a[2].split(" (")[0][:30])
    assert len(seen) >= 2


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
def test_roundtrip_matches_reference(oracle):
    rng = np.random.default_rng(5)
    for v in list(rng.uniform(-100, 100, 200)) + [0.1, 1.0, 3.0, 1e-20, 123456789.0]:
        for s in (repr(float(v)), f"{v:.25f}", f"{v:.3e}"):
            assert oracle.roundtrip(s) == oracle.roundtrip(s, "ref")


def _ladder_rows(q, dilation):
    return [dict(square_id=str(i), x=format(float(x) * dilation, ".17g"), y=format(float(y) * dilation, ".17g"),
                 angle=format(float(a), ".17g")) for i, (x, y, a) in enumerate(q)]


def test_candidate_ladders_match_golden(oracle):
    """certified_candidate / certify_q results of the reference (its saved
    search outputs and demo-test inputs) reproduced by the oracle certifier
    on the same dilated rows."""
    cands = json.loads((GOLDEN / "candidates.json").read_text())
    assert len(cands) == 9
    for c in cands:
        for key in ("candidate", "certify_q"):
            want = c[key]
            if "error" in want:
                continue
            ok, L, reason, _ = oracle.certify(c["n"], _ladder_rows(c["q"], want["dilation"]))
            assert ok and L == want["L"], (c["name"], key, reason)


def test_cpu_parallel_tempering_baseline(oracle):
    """The CPU annealer (the timed CPU baseline of the search workloads)
    shrinks a loose grid to a dilation-certified side below its start, its
    counters add up, and it is deterministic in its seed."""
    from types import SimpleNamespace as NS
    rng = np.random.default_rng(3)
    n, w = 9, 3
    xy = np.stack([np.arange(n) % w + 0.5, np.arange(n) // w + 0.5], 1) * 1.1
    xya = np.concatenate([xy, rng.uniform(0, 0.05, (n, 1))], 1)
    job = NS(xya=xya, replicas=4, sweeps=400, exchange_every=10, L0=3.3, tmin=1e-4, tmax=1e-2, sigma_xy=0.02,
             sigma_a=0.05, shrink=0.002, seed=7)
    (a,), used = oracle.ptsa_batch([job], threads=2)
    (b,), _ = oracle.ptsa_batch([job], threads=1)
    assert used == 1 and a == b
    assert a["proposals"] == 4 * 400 * n and 0 < a["accepted"] < a["proposals"]
    assert a["exchange_attempts"] > 0 and a["shrinks"] >= 1
    assert 3.0 <= a["best_L"] < 3.3
    many, used = oracle.ptsa_batch([job] * 3, threads=3)
    assert used == 3 and all(m == a for m in many)
