"""GPU interval certifier: verdict, reason, score and 50-decimal side equal
to the oracle (the reference certifier's algorithm) on the same strings, bit
for bit; and to the reference's own golden vectors."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _gpu(items, ctx, roundtrip=False):
    from sqs import core
    return core.evaluate_batch(items, roundtrip=roundtrip, ctx=ctx)


def _same(items, res, oracle, roundtrip=False):
    for (n, rows), (n2, score, L, reason) in zip(items, res):
        if roundtrip:
            rows = [dict(r, x=oracle.roundtrip(r["x"]), y=oracle.roundtrip(r["y"]),
                         angle=oracle.roundtrip(r["angle"])) for r in rows]
        ok, Lo, ro, so = oracle.certify(n, rows)
        assert (L is not None) == ok, (n, reason, ro)
        assert L == Lo, (n, L, Lo)
        assert reason == ro, (n, reason, ro)
        assert score == so, (n, score, so)


def test_golden_cases(ctx):
    cases = json.loads((GOLDEN / "certify_cases.json").read_text())
    res = _gpu([(c["n"], c["rows"]) for c in cases], ctx)
    for c, (n, score, L, reason) in zip(cases, res):
        assert (L is not None) == c["ok"], c["name"]
        assert L == c["L"], c["name"]
        assert reason == c["reason"], c["name"]
        assert score == c["score"], c["name"]


def test_corpus_matches_oracle(ctx, oracle):
    from sqs.workloads import certify_corpus
    items = certify_corpus(300, seed=5, n_hi=300, overlap_frac=0.15)
    _same(items, _gpu(items, ctx), oracle)


def test_angles_across_all_quadrants(ctx, oracle):
    # Angles up to the +-100 radian limit exercise every quadrant of the
    # pi/2 reduction (a quadrant error is invisible for |a| < pi/2 + pi/4
    # because a square turned by 90 degrees has the same corners).
    rng = np.random.default_rng(17)
    items = []
    for a in list(rng.uniform(-100, 100, 40)) + [-99.99, 99.99, 7.0, -7.0, 3.14159, -1.5707963]:
        items.append((1, [dict(square_id="0", x="0.5", y="0.5", angle=repr(float(a)))]))
        items.append((2, [dict(square_id="0", x="0.5", y="0.5", angle=repr(float(a))),
                          dict(square_id="1", x="2.0", y="0.5", angle=repr(float(-a / 3)))]))
    _same(items, _gpu(items, ctx), oracle)


def test_random_overlapping_and_shuffled(ctx, oracle):
    from sqs.workloads import rows_of
    rng = np.random.default_rng(3)
    items = []
    for k in range(120):
        n = int(rng.integers(1, 60))
        L = 1.2 * math.sqrt(n) + 1
        q = np.concatenate([rng.uniform(0, L, (n, 2)), rng.uniform(-6, 6, (n, 1))], axis=1)
        rows = rows_of(q, ".%dg" % int(rng.integers(3, 18)))
        if k % 3 == 0:
            rng.shuffle(rows)
        items.append((n, rows))
    _same(items, _gpu(items, ctx), oracle)


EDGE_LITERALS = [
    "0.5", " 0.5 ", "+0.5", ".5", "5.", "0005.5000", "1.5E0", "15e-1", "-0", "0.0", "0",
    "10000", "-10000", "10000.0000000000009094947017729282379150390625",
    "10000.00000000000090949470177292823791503906251", "-10000.0000000000009094947017729282379150390626",
    "1e4", "1.0000000000000001e4", "1e400", "-1e400", "1e-400", "nan", "inf", "", " ", "1.2.3", "1e", "e5",
    "0x10", "1,5", "1" + "0" * 99, "1." + "0" * 98, "-." , "+", "1e+0005", "0.000000000000000000000000000001",
]


def test_literal_edges(ctx, oracle):
    items = []
    for lit in EDGE_LITERALS:
        for field in ("x", "y", "angle"):
            rows = [dict(square_id="0", x="0.5", y="0.5", angle="0")]
            rows[0][field] = lit
            items.append((1, rows))
    for a in ("100", "-100", "100.00000000000000710542735760100185871124267578125",
              "100.000000000000007105427357601001858711242675781251", "1e2", "99.99999999999999999999"):
        items.append((1, [dict(square_id="0", x="0.5", y="0.5", angle=a)]))
    # envelope errors
    items.append((2, [dict(square_id="0", x="0.5", y="0.5", angle="0")]))
    items.append((2, [dict(square_id="0", x="0.5", y="0.5", angle="0"), dict(square_id="0", x="1.5", y="0.5", angle="0")]))
    items.append((2, [dict(square_id="0", x="0.5", y="0.5", angle="0"), dict(square_id="2", x="1.5", y="0.5", angle="0")]))
    items.append((2, [dict(square_id="1", x="1.5", y="0.5", angle="0"), dict(square_id="0", x="0.5", y="0.5", angle="0")]))
    _same(items, _gpu(items, ctx), oracle)


def test_roundtrip_flag(ctx, oracle):
    cases = {c["name"]: c for c in json.loads((GOLDEN / "certify_cases.json").read_text())}
    items = [(c["n"], c["rows"]) for name, c in cases.items()
             if name.startswith(("goebel", "transport", "strip", "grid", "tilted"))]
    _same(items, _gpu(items, ctx, roundtrip=True), oracle, roundtrip=True)


def _deep_pair(theta: str, k: int, sign: int):
    """Two squares at angle theta whose centres are the support distance
    + sign * 10^-k apart along the first square's axis, written with 95
    significant digits: forces the interval stages past 63 digits."""
    import mpmath as mp
    with mp.workdps(200):
        a = mp.mpf(theta)
        c, s = mp.cos(a), mp.sin(a)
        d = 1 + sign * mp.mpf(10) ** (-k)
        x1, y1 = 3 + d * c, 4 + d * s
        return [dict(square_id="0", x="3", y="4", angle=theta),
                dict(square_id="1", x=mp.nstr(x1, 95), y=mp.nstr(y1, 95), angle=theta)]


def test_escalation_stages(ctx, oracle):
    items = []
    for theta in ("0.5", "1.1", "0.25", "1.5"):
        for k in (9, 30, 60, 70, 80, 90, 120):
            for sign in (1, -1):
                items.append((2, _deep_pair(theta, k, sign)))
    res = _gpu(items, ctx)
    _same(items, res, oracle)
    reasons = {r[3] for r in res}
    assert "ok" in reasons and "infeasible: Squares overlap (certified)" in reasons


def test_python_api_mirror(ctx):
    from sqs import core
    assert core.certify(4, core.grid(4), ctx=ctx) == "2." + "0" * 50
    with pytest.raises(ValueError, match=r"^n=2: "):
        core.certify(2, [dict(square_id="0", x=".5", y=".5", angle="0"),
                         dict(square_id="1", x=".6", y=".5", angle="0")], ctx=ctx)
    report = core.score({2: core.grid(2), 3: [dict(square_id="0", x=".5", y=".5", angle="0")]}, max_n=4, ctx=ctx)
    assert report["accepted"] == 1 and report["rejected"] == 1 and report["missing"] == 2
    assert report["score"] == pytest.approx(sum(core.infeasible_score(n) for n in (1, 3, 4)) + (2 / math.sqrt(2) - 1))


def test_full_seed42_corpus_equals_reference(ctx, oracle):
    """The whole certifier batch of the benchmark -- 10,000 packings, n
    log-uniform in [5, 1000], grids, tilted near-contact lattices, injected
    overlaps, seed 42 -- certified on the GPU in one call: verdict, reason,
    score and 50-decimal side equal to the compiled reference certifier
    (certifier.cpp, evaluate_single_puzzle :738-912) on every packing, or to
    the oracle restatement where the reference was not compiled."""
    from sqs import core
    from sqs.workloads import certify_corpus
    items = certify_corpus(10000, seed=42)
    arrs = core.pack_batch(items)
    out = core.certify_arrays(*arrs, ctx=ctx)
    which = "ref" if oracle.ref_available() else "oracle"
    ok, score, Ls, reasons = oracle.certify_batch_text(*arrs, which=which)
    bad = []
    for p in range(len(items)):
        v = out[p]
        got = (int(v.ok), float(v.score), v.L.decode(), v.reason.decode())
        want = (int(ok[p]), float(score[p]), Ls[p], reasons[p])
        if got != want:
            bad.append((p, items[p][0], got, want))
    assert not bad, (len(bad), bad[:3])
    assert 0 < ok.sum() < len(items)
    assert max(n for n, _ in items) > 900
