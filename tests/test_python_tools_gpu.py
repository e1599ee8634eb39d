"""The reference's Python tools on the GPU path: optimize_packing (the
reference's own test expectations, tests/test_optimizer.py), the command
line's validate / score (against the compiled reference certifier with
--roundtrip on the same CSV), merge and export-kaggle."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
REF_CERT = ROOT / "oracle" / "_ref" / "certifier"


def _cli(*args):
    env = dict(os.environ, PYTHONPATH=str(ROOT / "squares-in-squares_b200"))
    return subprocess.run([sys.executable, "-m", "sqs.cli", *map(str, args)], capture_output=True, text=True,
                          env=env, timeout=600)


def test_optimizer_reference_expectations(ctx):
    from sqs.core import certify, grid
    from sqs.optimizer import optimize_packing, tilted_five
    assert 2.7071 < float(certify(5, tilted_five(), ctx=ctx)) < 2.7072
    rows, rep = optimize_packing(5, attempts=0, seed=7, ctx=ctx)
    assert float(certify(5, rows, ctx=ctx)) < 3 and rep["improvements"] == 1
    rows, rep = optimize_packing(2, attempts=1, maxiter=3, seed=42, ctx=ctx)
    assert float(certify(2, rows, ctx=ctx)) <= 2 and rep["attempts"] == 1
    rows, rep = optimize_packing(4, attempts=2, ctx=ctx)
    assert float(certify(4, rows, ctx=ctx)) == 2 and rep["attempts"] == 0
    bad = grid(2)
    bad[1]["x"] = bad[0]["x"]
    with pytest.raises(ValueError):
        optimize_packing(2, bad, attempts=0, ctx=ctx)
    with pytest.raises(ValueError):
        optimize_packing(5, attempts=-1, ctx=ctx)


def test_optimizer_improves_a_grid(ctx, oracle):
    from sqs.optimizer import optimize_packing
    rows, rep = optimize_packing(10, attempts=8, maxiter=250, seed=3, ctx=ctx)
    assert rep["attempts"] == 8 and rep["initial_L"] == 4.0
    assert rep["final_L"] < 4.0 and rep["improvements"] >= 1
    ok, L, reason, _ = oracle.certify(10, rows)
    assert ok and float(L) == rep["final_L"], reason


def _write_csv(path, puzzles):
    lines, rid = ["id,n,square_id,x,y,angle"], 0
    for n, rows in sorted(puzzles.items()):
        for r in rows:
            lines.append(f"{rid},{n},{r['square_id']},{r['x']},{r['y']},{r['angle']}")
            rid += 1
    path.write_text("\n".join(lines) + "\n")


def test_cli_score_validate_merge_export(tmp_path):
    from sqs.core import grid
    from sqs.workloads import rows_of, tilted_lattice
    puzzles = {n: grid(n) for n in range(1, 16) if n != 6}
    puzzles[9] = rows_of(tilted_lattice(9, 1e-13, 0.4))  # near-contact tilted lattice
    bad = [dict(r) for r in grid(12)]
    bad[3]["x"] = bad[2]["x"]
    puzzles[12] = bad
    csv = tmp_path / "sub.csv"
    _write_csv(csv, puzzles)
    r = _cli("score", csv, "--max-n", 20, "--report", tmp_path / "rep.json")
    assert r.returncode == 0, r.stderr
    mine = json.loads(r.stdout)
    if REF_CERT.exists():
        ref = json.loads(subprocess.run([str(REF_CERT), str(csv), "--max-n", "20", "--roundtrip"],
                                        capture_output=True, text=True, timeout=300).stdout)
        for k in ("accepted", "missing", "rejected"):
            assert mine[k] == ref[k], k
        assert abs(mine["score"] - ref["score"]) < 1e-12
    assert len(json.loads((tmp_path / "rep.json").read_text())["results"]) == 20
    assert _cli("validate", csv, "--max-n", 20).returncode == 2            # n=12 overlaps
    del puzzles[12]
    _write_csv(csv, puzzles)
    assert _cli("validate", csv, "--max-n", 20, "--require-complete").returncode == 2
    # merge: a second file with a better n=5 and a broken n=3
    from sqs.optimizer import tilted_five
    other = {5: tilted_five(), 3: [dict(r, x="0.5") for r in grid(3)]}
    csv2 = tmp_path / "b.csv"
    _write_csv(csv2, other)
    r = _cli("merge", csv, csv2, "--output", tmp_path / "m.csv")
    assert r.returncode == 0, r.stderr
    from sqs.core import read_submission
    merged = read_submission(tmp_path / "m.csv")
    assert merged[5][0]["x"] == other[5][0]["x"] and merged[3][0]["x"] == puzzles[3][0]["x"]
    # export: puzzles that survive the numeric transport keep their strings,
    # and the exported file validates (literally and after the transport)
    r = _cli("export-kaggle", csv, "--output", tmp_path / "k.csv")
    assert r.returncode == 0, r.stderr
    exported = read_submission(tmp_path / "k.csv")
    assert [(q["x"], q["y"], q["angle"]) for q in exported[7]] == [(q["x"], q["y"], q["angle"]) for q in puzzles[7]]
    r = _cli("validate", tmp_path / "k.csv", "--max-n", 15)
    assert r.returncode == 0, r.stderr
