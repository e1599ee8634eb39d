"""Certification gate backed by the GPU interval certifier.

Mirrors the reference's squares.core entry points for this path
(core.py:22-62, 105-118): ``check_n``, ``grid``, ``evaluate(n, rows) ->
(n, score, L | None, reason)``, ``certify(n, rows) -> L`` raising
``ValueError("n=<n>: <reason>")``, ``score(puzzles, max_n)``, plus the
batched forms that are the point of a GPU gate.  Rows are dicts of strings
with keys square_id, x, y, angle, exactly as the reference passes them.

Verdicts, reasons, scores and the 50-decimal side are those of the
reference's C++ certifier (cuda/certifier.cpp:738-912), which agrees with
the Python metric on verdict and side; reason wording follows certifier.cpp.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Iterable

import numpy as np

from . import _native as N

Packing = list[dict[str, str]]
Puzzles = dict[int, Packing]
MAX_N = 1000
CERT_ROUNDTRIP = 1


Verdict = N.Verdict

_CTX: N.Context | None = None


def _ctx(ctx: N.Context | None) -> N.Context:
    global _CTX
    if ctx is not None:
        return ctx
    if _CTX is None:
        _CTX = N.Context(0)
    return _CTX


def check_n(n: int) -> None:
    if not 1 <= n <= MAX_N:
        raise ValueError("n must be in 1..1000")


def grid(n: int) -> Packing:
    """Half-integer grid centres with integer pitch, zero rotation."""
    check_n(n)
    width = math.isqrt(n - 1) + 1
    return [dict(square_id=str(i), x=f"{i % width}.5", y=f"{i // width}.5", angle="0") for i in range(n)]


def infeasible_score(n: int) -> float:
    return math.ceil(math.sqrt(n)) / math.sqrt(n) - 1


def pack_batch(items: Iterable[tuple[int, Packing]]):
    """Flatten (n, rows) items into the C ABI's arrays."""
    n_of, row_start, sids, lits = [], [0], [], []
    for n, rows in items:
        n_of.append(int(n))
        for r in rows:
            try:
                sids.append(int(r["square_id"]))
            except (ValueError, TypeError):
                sids.append(-1)
            lits.extend((str(r["x"]), str(r["y"]), str(r["angle"])))
        row_start.append(len(sids))
    enc = [s.encode("utf-8", "surrogateescape") for s in lits]
    lens = np.fromiter((len(b) for b in enc), dtype=np.int64, count=len(enc))
    off = np.zeros(len(enc) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    return (np.asarray(n_of, np.int32), np.asarray(row_start, np.int64), np.asarray(sids, np.int32),
            b"".join(enc), off)


def certify_arrays(n_of, row_start, square_id, text: bytes, lit_off, *, roundtrip: bool = False,
                   ctx: N.Context | None = None):
    """Certify packed arrays; returns a ctypes array of Verdict."""
    count = len(n_of)
    out = (Verdict * max(1, count))()
    if count == 0:
        return out
    n_of = np.ascontiguousarray(n_of, np.int32)
    row_start = np.ascontiguousarray(row_start, np.int64)
    square_id = None if square_id is None else np.ascontiguousarray(square_id, np.int32)
    lit_off = np.ascontiguousarray(lit_off, np.int64)
    c = _ctx(ctx)
    N.check(N.lib().sqs_certify_batch(c.handle, count, n_of.ctypes.data, row_start.ctypes.data,
                                      None if square_id is None else square_id.ctypes.data, text or b"\0",
                                      lit_off.ctypes.data, CERT_ROUNDTRIP if roundtrip else 0, out))
    return out


def evaluate_batch(items: Iterable[tuple[int, Packing]], *, roundtrip: bool = False,
                   ctx: N.Context | None = None) -> list[tuple[int, float, str | None, str]]:
    """[(n, score, L | None, reason)] for every (n, rows), one GPU batch."""
    items = list(items)
    for n, _ in items:
        check_n(n)
    out = certify_arrays(*pack_batch(items), roundtrip=roundtrip, ctx=ctx)
    res = []
    for k, (n, _) in enumerate(items):
        v = out[k]
        res.append((n, v.score, v.L.decode() if v.ok else None, v.reason.decode()))
    return res


def evaluate(n: int, rows: Packing, *, ctx: N.Context | None = None) -> tuple[int, float, str | None, str]:
    check_n(n)
    return evaluate_batch([(n, rows)], ctx=ctx)[0]


def certify(n: int, rows: Packing, *, ctx: N.Context | None = None) -> str:
    """Return L as a 50-decimal string; refuse malformed/uncertified results."""
    _, _, side, reason = evaluate(n, rows, ctx=ctx)
    if side is None or reason != "ok":
        raise ValueError(f"n={n}: {reason}")
    return side


def score(puzzles: Puzzles, max_n: int = 1000, *, roundtrip: bool = False,
          ctx: N.Context | None = None) -> dict:
    """Score with grid penalties for absent or rejected puzzles (core.py:105-118)."""
    check_n(max_n)
    work = [(n, rows) for n, rows in sorted(puzzles.items()) if 1 <= n <= max_n]
    got = {r[0]: r for r in evaluate_batch(work, roundtrip=roundtrip, ctx=ctx)}
    results = [got.get(n, (n, infeasible_score(n), None, "missing from submission")) for n in range(1, max_n + 1)]
    return dict(
        score=sum(r[1] for r in results), max_n=max_n,
        accepted=sum(r[3] == "ok" for r in results),
        missing=sum(r[3] == "missing from submission" for r in results),
        rejected=sum(r[3] not in ("ok", "missing from submission") for r in results),
        results=[dict(n=n, score=s, L=side, reason=reason) for n, s, side, reason in results],
    )


# ------------------------------------------------------------ submissions
COLUMNS = ("id", "n", "square_id", "x", "y", "angle")


def read_submission(path) -> Puzzles:
    """Rows of a submission CSV as strings, grouped by n, in file order
    (core.py:38-50): header id,n,square_id,x,y,angle, six fields per row,
    consecutive ids from 0, 1 <= n <= 1000; ValueError otherwise."""
    import csv
    import io
    from pathlib import Path

    text = Path(path).read_text(encoding="utf-8")
    reader = csv.DictReader(io.StringIO(text))
    if tuple(reader.fieldnames or ()) != COLUMNS:
        raise ValueError("CSV header must be id,n,square_id,x,y,angle")
    puzzles: Puzzles = {}
    for i, row in enumerate(reader):
        if None in row or any(value is None for value in row.values()):
            raise ValueError(f"row {i + 2} has the wrong number of fields")
        if row["id"] != str(i):
            raise ValueError(f"row {i + 2} must have id {i}")
        try:
            n = int(row["n"])
        except ValueError:
            raise ValueError(f"Row {i + 2}: invalid n value: {row['n']!r}") from None
        if not 1 <= n <= MAX_N:
            raise ValueError(f"Row {i + 2}: n={n} out of range [1, {MAX_N}]")
        puzzles.setdefault(n, []).append(row)
    return puzzles


def _structure_error(n: int, rows: Packing) -> str | None:
    if len(rows) != n:
        return f"n={n}: expected {n} rows, got {len(rows)}"
    try:
        ids = {int(r["square_id"]) for r in rows}
    except (ValueError, TypeError):
        return f"n={n}: invalid square_id"
    if ids != set(range(n)):
        return f"n={n}: square_ids should be 0..{n - 1}"
    return None


def certify_all(puzzles: Puzzles, *, ctx: N.Context | None = None) -> dict[int, str]:
    """certify() of every puzzle in one GPU batch: {n: L}; the first failure
    (in n order) raises ValueError("n=<n>: <reason>")."""
    items = sorted(puzzles.items())
    out = {}
    for n, _, side, reason in evaluate_batch(items, ctx=ctx):
        if side is None or reason != "ok":
            raise ValueError(f"n={n}: {reason}")
        out[n] = side
    return out


def write_submission(path, puzzles: Puzzles, *, validate: bool = True, ctx: N.Context | None = None) -> None:
    """Certify (validate=True; structural checks only for constructions such
    as grid()) and atomically replace the CSV, rows by n then square id
    (core.py:65-102)."""
    import csv
    import os
    import tempfile
    from pathlib import Path

    for n, rows in puzzles.items():
        check_n(n)
        if not validate:
            err = _structure_error(n, rows)
            if err:
                raise ValueError(err)
    if validate:
        certify_all(puzzles, ctx=ctx)
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = None
    try:
        with tempfile.NamedTemporaryFile(mode="w", encoding="utf-8", newline="", dir=path.parent,
                                         prefix=f".{path.name}.", delete=False) as handle:
            tmp = Path(handle.name)
            writer = csv.DictWriter(handle, fieldnames=COLUMNS)
            writer.writeheader()
            index = 0
            for n, rows in sorted(puzzles.items()):
                for row in sorted(rows, key=lambda r: int(r["square_id"])):
                    writer.writerow(dict(id=index, n=n, square_id=row["square_id"], x=row["x"], y=row["y"],
                                         angle=row["angle"]))
                    index += 1
        os.replace(tmp, path)
    finally:
        if tmp is not None:
            tmp.unlink(missing_ok=True)


def merge_best(candidates: list[Puzzles], *, ctx: N.Context | None = None) -> Puzzles:
    """Certified smallest L per n over the candidate sets, original strings
    kept; invalid candidates never replace valid ones, ties keep the first
    (core.py:121-137).  All candidates are certified in one GPU batch."""
    from decimal import Decimal

    items = [(n, rows) for puzzles in candidates for n, rows in sorted(puzzles.items())]
    best: Puzzles = {}
    sides: dict[int, Decimal] = {}
    for (n, rows), (_, _, side, reason) in zip(items, evaluate_batch(items, ctx=ctx) if items else []):
        if reason != "ok" or side is None:
            continue
        length = Decimal(side)
        if n not in sides or length < sides[n]:
            sides[n] = length
            best[n] = [dict(r) for r in rows]
    return best


def _strtod(s: str) -> float:
    """C strtod of the longest numeric prefix (0.0 when there is none)."""
    import re

    m = re.match(r"\s*[+-]?(?:inf(?:inity)?|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)", s, re.IGNORECASE)
    if not m:
        return 0.0
    try:
        return float(m.group(0))
    except ValueError:  # an exponent too large for a double
        return math.copysign(math.inf, -1.0 if m.group(0).strip().startswith("-") else 1.0)


def roundtrip_literal(s: str) -> str:
    """A literal after a numeric CSV round trip (certifier.cpp:914-929): the
    double it parses to, written with the fewest of 15, 16, 17 significant
    digits that read back to the same double, with ".0" added to integers."""
    v = _strtod(s)
    out = ""
    for prec in (15, 16, 17):
        out = "%.*g" % (prec, v)
        if _strtod(out) == v:
            break
    if not any(c in out for c in ".eE"):
        out += ".0"
    return out


def kaggle_roundtrip(puzzles: Puzzles) -> Puzzles:
    """Every x, y, angle after the numeric CSV transport a hosted scorer
    applies before the metric (core.py:140-153, as emulated by the
    certifier's --roundtrip)."""
    return {n: [dict(r, x=roundtrip_literal(r["x"]), y=roundtrip_literal(r["y"]),
                     angle=roundtrip_literal(r["angle"])) for r in rows]
            for n, rows in puzzles.items()}


def prepare_kaggle(puzzles: Puzzles, dilation: str = "1.00000002", *, ctx: N.Context | None = None) -> Puzzles:
    """Keep puzzles that survive the numeric transport; dilate the centres of
    the others by `dilation` (at 80 digits, written with 60) so contact gaps
    open; every result must certify literally and after the transport
    (core.py:156-186).  Certification runs in GPU batches."""
    from decimal import Decimal, localcontext

    factor = Decimal(dilation)
    if not Decimal(1) < factor <= Decimal("1.001"):
        raise ValueError("dilation must be > 1 and <= 1.001")
    certify_all(puzzles, ctx=ctx)
    transported = kaggle_roundtrip(puzzles)
    survives = {n: reason == "ok" for n, _, _, reason in evaluate_batch(sorted(transported.items()), ctx=ctx)}
    prepared: Puzzles = {}
    for n, rows in sorted(puzzles.items()):
        if survives[n]:
            prepared[n] = [dict(r) for r in rows]
            continue
        with localcontext() as dc:
            dc.prec = 80
            prepared[n] = [dict(r, **{axis: format(Decimal(r[axis]) * factor, ".60g") for axis in ("x", "y")})
                           for r in rows]
    certify_all(prepared, ctx=ctx)
    certify_all(kaggle_roundtrip(prepared), ctx=ctx)
    return prepared
