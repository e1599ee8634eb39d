"""The drop-in executables' argument, environment and CSV checks, which run
before any GPU work: every violation the reference programs reject exits
with status 2 (packing.cu:769-775, seeded.cu:832-846 and its validated
environment variables, certifier.cpp:933-994)."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

BIN = Path(__file__).resolve().parents[1] / "squares-in-squares_b200" / "bin"


def _run(args, env=None, **kw):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, env=e, timeout=60, **kw)


@pytest.fixture(scope="module")
def built():
    for name in ("packing", "seeded", "certifier"):
        if not (BIN / name).exists():
            pytest.skip(f"{name} not built (python squares-in-squares_b200/build.py)")
    return BIN


def _seed(tmp_path, text):
    p = tmp_path / "seed.txt"
    p.write_text(text)
    return p


@pytest.mark.parametrize("prog", ["packing", "seeded"])
def test_search_argument_checks(built, tmp_path, prog):
    good = _seed(tmp_path, "2 2\n0.5 0.5 0\n1.5 0.5 0\n")
    out = tmp_path / "o.json"
    bad_args = [
        [],
        [good, 1, 1, 8, 1],                       # six arguments needed
        [good, -1, 1, 8, 1, out],
        [good, 100001, 1, 8, 1, out],
        [good, 1, 4097, 8, 1, out],
        [good, 1, 1, 12, 1, out],                 # chains not a multiple of 8
        [good, 1, 1, 4104, 1, out],
        [tmp_path / "missing.txt", 1, 1, 8, 1, out],
        [_seed(tmp_path, "1001 40\n"), 1, 1, 8, 1, out],
        [_seed(tmp_path, "2 65\n0.5 0.5 0\n1.5 0.5 0\n"), 1, 1, 8, 1, out],
        [_seed(tmp_path, "2 2\n0.5 0.5 0\n1.5 nan 0\n"), 1, 1, 8, 1, out],
        [_seed(tmp_path, "3 2\n0.5 0.5 0\n1.5 0.5 0\n"), 1, 1, 8, 1, out],   # too few rows
    ]
    for a in bad_args:
        r = _run([built / prog, *a])
        assert r.returncode == 2, (a, r.stdout, r.stderr)
        assert f"{prog}: " not in r.stderr, (a, r.stderr)  # rejected before any device work
    assert not out.exists()


@pytest.mark.parametrize("prog,var,value", [
    ("packing", "PACK_TMAX", "2"), ("packing", "PACK_MOVE", "0.5"), ("packing", "PACK_SHRINK", "x"),
    ("packing", "PACK_MAX_CHAINS", "4"), ("seeded", "SEED_TMAX", "0.2"), ("seeded", "SEED_POLISH", "5000"),
    ("seeded", "SEED_COLLECTIVE", "2"), ("seeded", "SEED_MOVE", "0.02x"), ("seeded", "SEED_QUENCH_ALL", "2"),
    ("packing", "PACK_CERT_ALL", "-1"), ("seeded", "SEED_QUENCH_STEPS", "-2"), ("packing", "PACK_QUENCH_STEPS", "3000")])
def test_search_environment_checks(built, tmp_path, prog, var, value):
    seed = _seed(tmp_path, "2 2\n0.5 0.5 0\n1.5 0.5 0\n")
    r = _run([built / prog, seed, 1, 1, 8, 1, tmp_path / "o.json"], env={var: value})
    assert r.returncode == 2 and f"invalid {var}" in r.stderr


def test_packing_tmax_below_tmin(built, tmp_path):
    seed = _seed(tmp_path, "2 2\n0.5 0.5 0\n1.5 0.5 0\n")
    r = _run([built / "packing", seed, 1, 1, 8, 1, tmp_path / "o.json"], env={"PACK_TMIN": "1e-3", "PACK_TMAX": "1e-4"})
    assert r.returncode == 2


@pytest.mark.parametrize("body", [
    "",                                                    # empty file
    "id,n,square_id,x,y\n0,1,0,0.5,0.5\n",                 # header
    "id,n,square_id,x,y,angle\n1,1,0,0.5,0.5,0\n",         # ids start at 0
    "id,n,square_id,x,y,angle\n0,1,0,0.5,0.5\n",           # five fields
    "id,n,square_id,x,y,angle\n0,1,0,0.5,0.5,0,7\n",       # seven fields
    "id,n,square_id,x,y,angle\n0,1001,0,0.5,0.5,0\n",      # n out of range
    "id,n,square_id,x,y,angle\n0,0,0,0.5,0.5,0\n",
])
def test_certifier_csv_checks(built, tmp_path, body):
    p = tmp_path / "s.csv"
    p.write_text(body)
    r = _run([built / "certifier", p])
    assert r.returncode == 2, r.stdout
    assert "certifier: " not in r.stderr, r.stderr  # rejected before any device work
    r = _run([built / "certifier"])
    assert r.returncode == 2
    r = _run([built / "certifier", tmp_path / "absent.csv"])
    assert r.returncode == 2
