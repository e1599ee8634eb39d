"""Standalone FP64 polish (sqs_polish_batch) and the dilation-ladder gates
that mirror the reference's polish.certify_q / polish.polish and
demo.certified_candidate, against the reference's own results on its saved
search outputs (tests/golden/candidates.json) and the oracle certifier."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _cands():
    return json.loads((GOLDEN / "candidates.json").read_text())


def _q(c):
    return [[float(v) for v in row] for row in c["q"]]


def test_certified_candidate_and_certify_q_match_reference(ctx):
    from sqs.demo import certified_candidate
    from sqs.polish import certify_q
    for c in _cands():
        raw = dict(n=c["n"], q=_q(c))
        for key, fn in (("candidate", lambda: certified_candidate(raw, ctx=ctx)),
                        ("certify_q", lambda: certify_q(raw["q"], ctx=ctx))):
            want = c[key]
            if "error" in want:
                with pytest.raises(ValueError, match=want["error"]):
                    fn()
                continue
            rows, side, dil = fn()
            assert dil == want["dilation"] and side == want["side"], (c["name"], key)
            assert len(rows) == c["n"]


def test_polish_keeps_or_improves_and_certifies(ctx, oracle):
    from sqs.polish import certify_q, polish, polish_batch
    raws = [c for c in _cands() if c["name"].startswith("raw")]
    qs = [np.array(_q(c)) for c in raws]
    res = polish_batch(qs, 300, ctx=ctx)
    for c, q, (p, info) in zip(raws, qs, res):
        assert info["L_in"] < 1e29 and info["L_out"] <= info["L_in"]
        assert 0 < info["iterations"] <= 300
        rows, side, _ = certify_q(p, ctx=ctx)
        ok, L, reason, _ = oracle.certify(c["n"], rows)
        assert ok and float(L) == side, reason
        # the certified side of the polished state is within the FP64 bound
        assert side <= info["L_out"] * (1 + 1e-6) + 1e-12
    # the single-state mirror returns the better of polished and input
    rows, rep = polish(qs[0], 300, ctx=ctx)
    assert rep["n"] == 5 and rep["L"] <= raws[0]["certify_q"]["side"] + 1e-12


def test_polish_resolves_overlapping_input(ctx, oracle):
    from sqs.core import grid
    from sqs.polish import certify_q, polish_batch
    n = 16
    g = np.array([[float(r["x"]), float(r["y"]), float(r["angle"])] for r in grid(n)])
    squeezed = g.copy()
    squeezed[:, :2] *= 0.96          # 4% overlaps: beyond the 0.8% dilation bound
    p, info = polish_batch([squeezed], 2000, ctx=ctx)[0]
    assert info["L_in"] >= 1e29 and info["L_out"] < 1e29
    rows, side, _ = certify_q(p, ctx=ctx)
    assert oracle.certify(n, rows)[0]
    assert side < 4.05


def test_polish_batch_is_deterministic_and_ragged(ctx):
    from sqs.polish import polish_batch
    from sqs.anneal import jittered_grid
    qs = [jittered_grid(n, seed=n)[0] for n in (1, 2, 7, 30, 130)]
    a = polish_batch(qs, 200, ctx=ctx)
    b = polish_batch(qs[::-1], 200, ctx=ctx)[::-1]
    for (pa, ia), (pb, ib) in zip(a, b):
        assert np.array_equal(pa, pb) and ia == ib
        assert ia["L_out"] <= ia["L_in"] and ia["L_out"] < 1e29  # jittered grids may start overlapped
    # one square: the polish turns it toward angle 0, side toward 1
    assert 1.0 <= a[0][1]["L_out"] < a[0][1]["L_in"]


def test_polish_errors(ctx):
    from sqs import SQSError
    from sqs.polish import polish_batch
    with pytest.raises(ValueError):
        polish_batch([np.array([[0.5, 0.5, float("nan")]])], ctx=ctx)
    with pytest.raises(ValueError):
        polish_batch([np.zeros((1001, 3))], ctx=ctx)
    with pytest.raises(SQSError):
        polish_batch([np.array([[0.5, 0.5, 0.0]])], -1, ctx=ctx)
    assert polish_batch([], ctx=ctx) == []
