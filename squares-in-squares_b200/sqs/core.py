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
