"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run with $SQS_REFERENCE naming a checkout of the reference sources (there is
no default) and the compiled reference in oracle/_ref:

    make -C oracle ref REF=$SQS_REFERENCE && python tests/golden/make_golden.py

Outputs (committed):
  certify_cases.json  packings with the verdict, reason and 50-decimal side
                      from the reference's Python metric (core.evaluate) and
                      from its C++ certifier (certifier.cpp); the two agree on
                      every case kept here.
  sat_pairs.json      random unit-square pairs with the reference's FP64
                      pair() energy and gradient (seeded.cu:92) and boundary()
                      (seeded.cu:96) values, computed by oracle/_ref.
  optimizer.json      the rows of the reference's n = 5 construction
                      (squares.optimizer.tilted_five, optimizer.py:13-35).
  candidates.json     the reference's saved search outputs (cuda/results/
                      raw{5,10,11,17,50}.json: n and the raw state q) and the
                      test inputs of tests/test_cuda_demo.py, with the result
                      of its certified_candidate (demo.py:25-40) and certify_q
                      (polish.py:52-65): the 50-decimal side and the dilation,
                      or the ValueError message.
"""
from __future__ import annotations

import json
import os
import sys
from decimal import Decimal
from pathlib import Path

import numpy as np

if not os.environ.get("SQS_REFERENCE"):
    sys.exit("make_golden.py: set SQS_REFERENCE to a checkout of the reference sources")
REF = Path(os.environ["SQS_REFERENCE"])
HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(REF / "src"))
sys.path.insert(0, str(REF / "cuda"))
sys.path.insert(0, str(ROOT / "oracle"))

from squares.core import evaluate, grid, kaggle_roundtrip, prepare_kaggle  # noqa: E402
from squares.optimizer import tilted_five  # noqa: E402
from scheduler import goebel, strip_construction  # noqa: E402
import demo  # noqa: E402
import polish as ref_polish  # noqa: E402
import oracle as O  # noqa: E402


def pair_rows(x):
    return [dict(square_id="0", x=".5", y=".5", angle="0"),
            dict(square_id="1", x=x, y=".5", angle="0")]


def cases():
    out = []

    def add(name, n, rows):
        out.append(dict(name=name, n=n, rows=[dict(square_id=str(r["square_id"]), x=str(r["x"]),
                                                    y=str(r["y"]), angle=str(r["angle"])) for r in rows]))

    for n in (1, 2, 3, 4, 5, 9, 10, 16, 31, 100):
        add(f"grid{n}", n, grid(n))
    for a in (1, 2, 4, 5):
        rows = goebel(a)
        add(f"goebel{a}", len(rows), rows)
    for k in (2, 3, 4, 7):
        rows = strip_construction(k)
        add(f"strip{k}", len(rows), rows)
    add("tilted_five", 5, tilted_five())
    for x in ("1.5", "1.499999999999999999999999999999", "1.500000000000000000000000000001", ".6", "2.5"):
        add(f"contact_{x}", 2, pair_rows(x))
    for field, value in (("x", "sqrt(2)"), ("y", "nan"), ("x", "1e400"), ("x", "10001"),
                         ("angle", "101"), ("x", "1." + "0" * 101)):
        rows = grid(1)
        rows[0][field] = value
        add(f"limit_{field}_{value[:12]}", 1, rows)
    rows = grid(2)
    rows[1]["square_id"] = "0"
    add("duplicate_id", 2, rows)
    add("wrong_count", 3, grid(2))
    # goebel(2) loses its 1e-40 dilation in the float transport; the
    # prepared copy survives it.
    raw = {10: goebel(2)}
    add("goebel2_transported", 10, kaggle_roundtrip(raw)[10])
    add("goebel2_prepared", 10, prepare_kaggle(raw)[10])
    rows = [dict(square_id="0", x="0.10000000000000001", y="0", angle="0"),
            dict(square_id="1", x="1.100000000000000010000000000001", y="0", angle="0")]
    add("transport_gap", 2, rows)
    add("transport_gap_transported", 2, kaggle_roundtrip({2: rows})[2])
    # The reference's saved GPU outputs after its dilation ladder.
    for n in (5, 10, 11, 17, 50):
        rawj = json.loads((REF / "cuda" / "results" / f"raw{n}.json").read_text())
        rows, _, _ = demo.certified_candidate(rawj)
        add(f"gpu_raw{n}_certified", n, rows)
    # Rotated pairs near contact: a gap of 10^-k along the first square's axis.
    rng = np.random.default_rng(2024)
    for k in (3, 6, 9, 12, 20, 30):
        for sign in (+1, -1):
            a1, a2 = rng.uniform(0, 1.5, 2)
            c, s = np.cos(a1), np.sin(a1)
            # centre offset along square 1's x axis: separated by exactly the
            # support distance plus sign * 10^-k (computed in Decimal by the metric)
            r = 0.5 + 0.5 * (abs(np.cos(a2 - a1)) + abs(np.sin(a2 - a1)))
            d = Decimal(repr(float(r))) + sign * Decimal(10) ** -k
            rows = [dict(square_id="0", x="3", y="4", angle=repr(float(a1))),
                    dict(square_id="1", x=str(Decimal(3) + d * Decimal(repr(float(c)))),
                         y=str(Decimal(4) + d * Decimal(repr(float(s)))), angle=repr(float(a2)))]
            add(f"tilted_pair_1e-{k}_{'gap' if sign > 0 else 'overlap'}", 2, rows)
    return out


def main():
    if not O.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    kept = []
    for c in cases():
        n, rows = c["n"], c["rows"]
        _, score, side, reason = evaluate(n, rows)
        ok_ref, L_ref, reason_ref, score_ref = O.certify(n, rows, "ref")
        # Reason wording differs between the Python metric and certifier.cpp;
        # the verdict and side must agree.
        assert (reason == "ok") == ok_ref, (c["name"], reason, reason_ref)
        assert side == L_ref, (c["name"], side, L_ref)
        c.update(ok=ok_ref, L=L_ref, reason=reason_ref, score=score_ref, metric_reason=reason)
        kept.append(c)
    (HERE / "certify_cases.json").write_text(json.dumps(kept, indent=1) + "\n")

    rng = np.random.default_rng(832)
    P = rng.uniform(-1, 1, (600, 2, 3))
    recs = []
    ref = O.ref_seeded()
    import ctypes as C
    dp = C.POINTER(C.c_double)
    for p, q in P:
        g = np.zeros(3)
        pp, qq = np.ascontiguousarray(p), np.ascontiguousarray(q)
        e = ref.ref_pair(pp.ctypes.data_as(dp), qq.ctypes.data_as(dp), g.ctypes.data_as(dp))
        gb = np.zeros(3)
        b = ref.ref_boundary(pp.ctypes.data_as(dp), 1.3, gb.ctypes.data_as(dp))
        recs.append(dict(p=p.tolist(), q=q.tolist(), e=e, g=g.tolist(), wall_L=1.3, wall=b, wall_g=gb.tolist()))
    (HERE / "sat_pairs.json").write_text(json.dumps(recs) + "\n")

    cands = []
    for n in (5, 10, 11, 17, 50):
        raw = json.loads((REF / "cuda" / "results" / f"raw{n}.json").read_text())
        cands.append(dict(name=f"raw{n}", n=n, q=raw["q"]))
    cands += [dict(name="separated_pair", n=2, q=[[.5, .5, 0], [1.5, .5, 0]]),
              dict(name="empty", n=2, q=[]),
              dict(name="coincident", n=2, q=[[.5, .5, 0], [.5, .5, 0]]),
              dict(name="nan", n=2, q=[[float("nan"), 0, 0], [1, 0, 0]])]
    for c in cands:
        raw = dict(n=c["n"], q=c["q"])
        try:
            rows, side, dil = demo.certified_candidate(raw)
            c["candidate"] = dict(L=str(demo.certify(c["n"], rows)), side=side, dilation=dil)
        except ValueError as e:
            c["candidate"] = dict(error=str(e))
        try:
            rows, side, dil = ref_polish.certify_q(c["q"])
            c["certify_q"] = dict(L=str(demo.certify(c["n"], rows)), side=side, dilation=dil)
        except ValueError as e:
            c["certify_q"] = dict(error=str(e))
    (HERE / "optimizer.json").write_text(json.dumps(dict(tilted_five=tilted_five()), indent=1) + "\n")
    (HERE / "candidates.json").write_text(json.dumps(cands, indent=1).replace("NaN", "\"nan\"") + "\n")
    print(f"{len(kept)} certifier cases, {len(recs)} SAT pairs, {len(cands)} candidates")


if __name__ == "__main__":
    main()
