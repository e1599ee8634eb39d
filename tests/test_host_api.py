"""Host-side parts of the Python mirror that need no GPU: the n = 5
construction against the reference's own rows, the numeric round trip of
literals against the compiled reference certifier, submission CSV reading
and writing, and the command line's grid baseline and argument checks."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"


def test_tilted_five_rows_match_reference():
    from sqs.optimizer import tilted_five_rows
    want = json.loads((GOLDEN / "optimizer.json").read_text())["tilted_five"]
    assert tilted_five_rows() == want


def test_roundtrip_literal_matches_reference(oracle):
    from sqs.core import roundtrip_literal
    which = "ref" if oracle.ref_available() else "oracle"
    rng = np.random.default_rng(11)
    cases = ["0", "0.5", "1", "-2", "1.5", "0.1", "3.70986129358606842598315732926024052282460003136629",
             "1e-5", "1E+3", "123456789012345678", "0.30000000000000004", "-0.0", "7.", ".25", "1e400",
             "2.5e-320", "12abc", "abc", " 4.5", "+3.25"]
    cases += [repr(float(v)) for v in rng.uniform(-50, 50, 200)]
    cases += [format(float(v), ".25g") for v in rng.uniform(0, 10, 200)]
    for s in cases:
        assert roundtrip_literal(s) == oracle.roundtrip(s, which), s


def _csv(tmp_path, body):
    p = tmp_path / "s.csv"
    p.write_text(body)
    return p


def test_read_submission(tmp_path):
    from sqs.core import read_submission
    p = _csv(tmp_path, "id,n,square_id,x,y,angle\n0,1,0,0.5,0.5,0\n1,2,1,1.5,0.5,0\n2,2,0,0.5,0.5,0\n")
    got = read_submission(p)
    assert list(got) == [1, 2] and [r["square_id"] for r in got[2]] == ["1", "0"]
    assert got[2][0]["x"] == "1.5"  # strings, file order
    for body in ("id,n,square_id,x,y\n", "id,n,square_id,x,y,angle\n1,1,0,0.5,0.5,0\n",
                 "id,n,square_id,x,y,angle\n0,1,0,0.5,0.5\n", "id,n,square_id,x,y,angle\n0,1001,0,0.5,0.5,0\n",
                 "id,n,square_id,x,y,angle\n0,x,0,0.5,0.5,0\n"):
        with pytest.raises(ValueError):
            read_submission(_csv(tmp_path, body))


def test_write_submission_grid_roundtrip(tmp_path):
    from sqs.core import grid, read_submission, write_submission
    puzzles = {n: grid(n) for n in (1, 3, 7)}
    out = tmp_path / "sub" / "g.csv"
    write_submission(out, puzzles, validate=False)
    back = read_submission(out)
    assert back.keys() == puzzles.keys()
    for n in puzzles:
        assert [(r["square_id"], r["x"], r["y"], r["angle"]) for r in back[n]] == \
               [(r["square_id"], r["x"], r["y"], r["angle"]) for r in puzzles[n]]
    bad = {2: grid(2)[:1]}
    with pytest.raises(ValueError):
        write_submission(tmp_path / "b.csv", bad, validate=False)
    assert not (tmp_path / "b.csv").exists()


def _cli(*args):
    env = dict(os.environ, PYTHONPATH=str(ROOT / "squares-in-squares_b200"))
    return subprocess.run([sys.executable, "-m", "sqs.cli", *map(str, args)], capture_output=True, text=True,
                          env=env, timeout=120)


def test_cli_baseline_and_argument_errors(tmp_path):
    import math
    out = tmp_path / "base.csv"
    r = _cli("baseline", "--max-n", 12, "--output", out)
    assert r.returncode == 0, r.stderr
    rep = json.loads(r.stdout)
    assert rep["puzzles"] == 12 and rep["rows"] == 78
    assert math.isclose(rep["score"], sum(math.ceil(math.sqrt(n)) / math.sqrt(n) - 1 for n in range(1, 13)))
    assert out.read_text().startswith("id,n,square_id,x,y,angle\n0,1,0,0.5,0.5,0\n")
    assert _cli("baseline", "--max-n", 0).returncode == 2
    assert _cli("optimize", "--n", 5).returncode == 2          # --output required
    bad = _csv(tmp_path, "id,n,x\n")
    r = _cli("score", bad)
    assert r.returncode == 2 and "error:" in r.stderr
