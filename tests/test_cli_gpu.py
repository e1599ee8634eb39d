"""The drop-in executables on the GPU: `certifier` prints the same summary
and per-n details as the reference's compiled certifier on the same CSV, and
`packing` / `seeded` write the reference's raw-JSON report whose best state
passes the official gate (demo.certified_candidate)."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "squares-in-squares_b200" / "bin"
REF_CERT = ROOT / "oracle" / "_ref" / "certifier"

# Keys of the reference's raw JSON (packing.cu:860-864, seeded.cu:949-969).
PACKING_KEYS = ["n", "target_L", "seconds", "chain_steps", "proposals", "feasible_checkpoints", "shrinks", "chains",
                "sm_count", "blocks_per_sm", "wave_chains", "device", "q"]
SEEDED_KEYS = ["n", "target_L", "seconds", "shrinks", "epochs", "steps", "chains", "device", "sm_count",
               "blocks_per_sm", "wave_chains", "collective", "polish", "structured", "proposals", "accepted",
               "exchange_attempts", "exchange_accepts", "q"]


def _csv(tmp_path):
    from sqs.core import grid
    from sqs.workloads import rows_of, tilted_lattice
    lines = ["id,n,square_id,x,y,angle"]
    rid = 0

    def put(n, rows):
        nonlocal rid
        for r in rows:
            lines.append(f"{rid},{n},{r['square_id']},{r['x']},{r['y']},{r['angle']}")
            rid += 1

    for n in range(1, 31):
        if n == 7:
            continue                                   # missing
        rows = grid(n)
        if n == 5:                                     # overlap
            rows = [dict(r) for r in rows]
            rows[1]["x"] = "1.4999999999"
        if n == 9:                                     # shuffled square ids
            rows = rows[::-1]
        put(n, rows)
    for n, gap, theta in ((33, 1e-9, 0.3), (34, 1e-13, 0.5)):
        put(n, rows_of(tilted_lattice(n, gap, theta)))
    put(35, [dict(square_id=str(i), x=repr(0.5 + i), y="0.5", angle="0.1") for i in range(35)])  # walls
    p = tmp_path / "sub.csv"
    p.write_text("\n".join(lines) + "\n")
    return p


def _cmp(a: dict, b: dict):
    for k in ("seconds", "threads"):
        a.pop(k, None)
        b.pop(k, None)
    assert a == b


@pytest.mark.parametrize("extra", [[], ["--roundtrip"], ["--max-n", "20"]])
def test_certifier_cli_matches_reference(tmp_path, extra):
    if not REF_CERT.exists():
        pytest.skip("compiled reference certifier absent (make -C oracle ref)")
    csv = _csv(tmp_path)
    mine = subprocess.run([str(BIN / "certifier"), str(csv), *extra, "--details", str(tmp_path / "a.json")],
                          capture_output=True, text=True, timeout=300)
    ref = subprocess.run([str(REF_CERT), str(csv), *extra, "--threads", "4", "--details", str(tmp_path / "b.json")],
                         capture_output=True, text=True, timeout=300)
    assert mine.returncode == 0 and ref.returncode == 0, (mine.stderr, ref.stderr)
    _cmp(json.loads(mine.stdout), json.loads(ref.stdout))
    da, db = json.loads((tmp_path / "a.json").read_text()), json.loads((tmp_path / "b.json").read_text())
    _cmp(da, db)
    s = json.loads(mine.stdout)
    assert s["missing"] >= 1 and s["rejected"] >= 1 and s["accepted"] >= 15


def _seed_file(tmp_path, n, seed):
    # the grid at pitch 1.05 in a container of 1.05 ceil(sqrt n): feasible,
    # with room for the search to find certified states below the seed side
    from sqs.anneal import jittered_grid
    xya, L = jittered_grid(n, jitter=0.0, angle_hi=1e-9, seed=seed)
    xya[:, :2] *= 1.05
    L *= 1.05
    p = tmp_path / f"seed{n}.txt"
    p.write_text(f"{n} {L}\n" + "".join(f"{x:.17g} {y:.17g} {a:.17g}\n" for x, y, a in xya))
    return p, L


@pytest.mark.parametrize("prog,keys", [("seeded", SEEDED_KEYS), ("packing", PACKING_KEYS)])
def test_search_cli_report_passes_the_official_gate(tmp_path, oracle, prog, keys):
    from sqs.demo import certified_candidate
    seed, L = _seed_file(tmp_path, 10, 42)
    out = tmp_path / "raw.json"
    env = {"SEED_POLISH": "100"} if prog == "seeded" else {"PACK_TMIN": "1e-6", "PACK_TMAX": "1e-2"}
    import os
    e = dict(os.environ)
    e.update(env)
    r = subprocess.run([str(BIN / prog), str(seed), "40", "64", "16", "7", str(out)], capture_output=True, text=True,
                       timeout=600, env=e)
    assert r.returncode == 0, r.stderr
    raw = json.loads(out.read_text())
    assert list(raw) == keys
    assert raw["n"] == 10 and raw["chains"] == 16 and raw["proposals"] > 0
    assert raw["target_L"] < L
    if prog == "seeded":
        assert raw["polish"] == 100 and raw["epochs"] == 40 and raw["steps"] == 64
    else:
        assert raw["chain_steps"] == 16 * 40 * 64
    q = np.asarray(raw["q"])
    assert q.shape == (10, 3)
    rows, side, dil = certified_candidate(raw)
    ok, Ls, reason, _ = oracle.certify(10, rows)
    assert ok and float(Ls) == side, reason
    assert side <= raw["target_L"] * dil * (1 + 1e-9)
