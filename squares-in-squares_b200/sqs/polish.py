"""FP64 gradient polish on the GPU and the dilation ladder that turns a raw
state into an officially certified packing.

Mirrors the reference's cuda/polish.py: ``certify_q(q)`` (polish.py:52-65)
and ``polish(q, maxiter)`` (polish.py:67-107), which returns ``(rows,
report)`` and raises ``ValueError`` when nothing certifies.  The reference
polishes with SLSQP on the CPU and only for n <= 50; here every packing of a
batch is polished by one CTA of the sqs_polish_batch kernel (n <= 1000), and
every rung of a dilation ladder is certified in one GPU certifier batch (the
first rung that passes is the result, as the reference's loop returns it).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .core import _ctx, evaluate_batch

CERTIFY_Q_LADDER = (1 + 1e-10, 1 + 1e-9, 1 + 1e-8, 1 + 1e-7, 1 + 1e-6)


def rows_of(q: np.ndarray, dilation: float = 1.0) -> list[dict[str, str]]:
    """Packing rows of a raw (n, 3) state with centres scaled by `dilation`,
    every value written with 17 significant digits (polish.py:58-60)."""
    return [dict(square_id=str(i), x=format(float(x) * dilation, ".17g"), y=format(float(y) * dilation, ".17g"),
                 angle=format(float(a), ".17g")) for i, (x, y, a) in enumerate(q)]


def _valid(q) -> np.ndarray:
    q = np.asarray(q, dtype=float)
    if q.ndim != 2 or q.shape[1] != 3 or not np.isfinite(q).all():
        raise ValueError("invalid coordinates")
    return q


def ladder_certify(qs: list[np.ndarray], ladder, *, ctx: N.Context | None = None):
    """For each state, the first rung of `ladder` whose dilated rows certify:
    [(rows, L, dilation) | None], all rungs of all states in one batch."""
    items = [(len(q), rows_of(q, d)) for q in qs for d in ladder]
    res = evaluate_batch(items, ctx=ctx) if items else []
    out = []
    for k, q in enumerate(qs):
        got = None
        for r, d in enumerate(ladder):
            n, _, L, _ = res[k * len(ladder) + r]
            if L is not None:
                got = (items[k * len(ladder) + r][1], float(L), d)
                break
        out.append(got)
    return out


def certify_q(q, *, ctx: N.Context | None = None):
    """(rows, L, dilation) of the first centre dilation 1 + 1e-10 .. 1 + 1e-6
    under which the state certifies; ValueError otherwise."""
    q = _valid(q)
    got = ladder_certify([q], CERTIFY_Q_LADDER, ctx=ctx)[0]
    if got is None:
        raise ValueError("official interval certification failed")
    return got


def polish_batch(qs: list, iters: int = 400, *, ctx: N.Context | None = None) -> list[tuple[np.ndarray, dict]]:
    """Polish every (n, 3) state on the GPU (sqs_polish_batch): returns
    [(polished state, {L_in, L_out, iterations, improved})]."""
    qs = [_valid(q) for q in qs]
    if not qs:
        return []
    for q in qs:
        if not 1 <= len(q) <= 1000:
            raise ValueError("polish supports n=1..1000")
    c = _ctx(ctx)
    n_of = np.array([len(q) for q in qs], dtype=np.int32)
    flat = np.ascontiguousarray(np.concatenate(qs, axis=0), dtype=np.float64)
    out = np.empty_like(flat)
    res = (N.PolishResult * len(qs))()
    N.check(N.lib().sqs_polish_batch(c.handle, len(qs), n_of.ctypes.data_as(C.POINTER(C.c_int32)),
                                     flat.ctypes.data_as(C.POINTER(C.c_double)), int(iters),
                                     out.ctypes.data_as(C.POINTER(C.c_double)), res))
    ans, r0 = [], 0
    for k, q in enumerate(qs):
        r = res[k]
        ans.append((out[r0:r0 + len(q)].copy(), dict(L_in=r.L_in, L_out=r.L_out, iterations=int(r.iterations),
                                                     improved=bool(r.improved))))
        r0 += len(q)
    return ans


def polish(q, maxiter: int = 400, *, ctx: N.Context | None = None):
    """Polish one state and certify the better of the polished and the input
    state: (rows, report) with report {n, L, dilation, iterations, converged,
    message}; ValueError when neither certifies (polish.py:67-107)."""
    q = _valid(q)
    n = len(q)
    polished, info = polish_batch([q], maxiter, ctx=ctx)[0]
    cands = ladder_certify([polished, q], CERTIFY_Q_LADDER, ctx=ctx)
    best = None
    for c in cands:
        if c is not None and (best is None or c[1] < best[1]):
            best = c
    if best is None:
        raise ValueError("official interval certification failed")
    rows, side, dilation = best
    return rows, dict(n=n, L=side, dilation=dilation, iterations=info["iterations"],
                      converged=bool(info["L_out"] < 1e29), message="improved" if info["improved"] else "kept",
                      L_polished=info["L_out"], L_input=info["L_in"])
