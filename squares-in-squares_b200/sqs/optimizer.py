"""Certified packing search behind the reference's optimizer interface.

Mirrors squares.optimizer (optimizer.py:13-118): ``tilted_five()`` and
``optimize_packing(n, initial=None, *, attempts=20, seed=42, maxiter=250)
-> (rows, report)``.  The reference refines the incumbent with L-BFGS-B
restarts on the CPU (n <= 50); here the attempts are parallel-tempering
jobs of the batched GPU annealer, started from the incumbent at a side a
little below it, with FP64 polish and the GPU interval certifier as the
acceptance gate, all attempts in one batched call.  Same argument checks,
the same n = 5 construction, the same report fields; the GPU search lifts
the n <= 50 limit of the CPU heuristic (n <= 1000).
"""
from __future__ import annotations

import math
from decimal import Decimal, localcontext

from . import _native as N
from .core import Packing, certify, check_n, evaluate_batch, grid


def _pi(prec: int) -> Decimal:
    """pi to `prec` digits by Machin's formula, pi = 16 atan(1/5) - 4 atan(1/239)."""
    with localcontext() as dc:
        dc.prec = prec + 10

        def atan_inv(k: int) -> Decimal:
            x = Decimal(1) / k
            x2, term, total, m = x * x, x, x, 1
            while True:
                term *= -x2
                m += 2
                step = term / m
                if step == 0 or abs(step) < Decimal(10) ** -(prec + 8):
                    break
                total += step
            return total

        return +(16 * atan_inv(5) - 4 * atan_inv(239))


def _nstr(v: Decimal, digits: int) -> str:
    """v with `digits` significant digits, trailing zeros dropped."""
    with localcontext() as dc:
        dc.prec = digits
        s = format(+v, "f")
    if "." in s:
        s = s.rstrip("0").rstrip(".")
    return s


def tilted_five_rows() -> Packing:
    """n = 5: four corner squares and a central square at 45 degrees in a side
    of 2 + 1/sqrt 2, centres dilated by 1.000000001 (the construction credited
    to Frits Goebel, 1979), written with 55 significant digits."""
    with localcontext() as dc:
        dc.prec = 60
        side = 2 + 1 / Decimal(2).sqrt()
        f = Decimal("1.000000001")
        h = Decimal("0.5")
        centres = [(h, h, Decimal(0)), (side - h, h, Decimal(0)), (h, side - h, Decimal(0)),
                   (side - h, side - h, Decimal(0)), (side / 2, side / 2, _pi(60) / 4)]
        return [dict(square_id=str(i), x=_nstr(x * f, 55), y=_nstr(y * f, 55), angle=_nstr(a, 55))
                for i, (x, y, a) in enumerate(centres)]


def tilted_five() -> Packing:
    """tilted_five_rows(), certified (optimizer.py:13-35)."""
    rows = tilted_five_rows()
    certify(5, rows)
    return rows


def optimize_packing(n: int, initial: Packing | None = None, *, attempts: int = 20, seed: int = 42,
                     maxiter: int = 250, ctx: N.Context | None = None) -> tuple[Packing, dict]:
    """Improve a certified packing of n squares (the grid by default): every
    attempt anneals the incumbent, compressed to a side 0.2% (every fifth
    attempt 1%) below it and perturbed by a shrinking amount, for
    20 * maxiter sweeps of 8 replicas, polishes and certifies its best state;
    a certified side below the incumbent's replaces it.  Returns the best
    rows and {n, seed, attempts, converged, initial_L, final_L,
    improvements}; raises ValueError for an uncertifiable warm start."""
    import numpy as np

    from .anneal import AnnealJob, anneal_batch

    check_n(n)
    if attempts < 0 or maxiter < 1:
        raise ValueError("attempts must be nonnegative and maxiter positive")
    rows = [dict(r) for r in (initial if initial is not None else grid(n))]
    side = float(certify(n, rows, ctx=ctx))
    start_side = side
    improvements = 0
    if n == 5:
        tilted = tilted_five()
        cand = float(certify(5, tilted, ctx=ctx))
        if cand < side:
            rows, side = tilted, cand
            improvements += 1
    completed = converged = 0
    if attempts > 0 and side > math.sqrt(n) + 1e-12:
        rng = np.random.default_rng(seed)
        q0 = np.array([[float(r[k]) for k in ("x", "y", "angle")] for r in
                       sorted(rows, key=lambda r: int(r["square_id"]))])
        q0[:, :2] -= q0[:, :2].min(axis=0) - 0.5
        jobs = []
        for a in range(attempts):
            temperature = 0.15 * (1 - a / max(attempts, 1)) + 0.005
            target = side - (0.01 if a % 5 == 0 else 0.002)
            q = q0.copy()
            if a:
                q += rng.normal(0, temperature * 0.1, q.shape)
            q[:, :2] *= target / side
            jobs.append(AnnealJob(q, L0=max(target, math.sqrt(n) + 1e-6), replicas=8, sweeps=20 * maxiter,
                                  exchange_every=10, tmin=1e-6, tmax=1e-2, seed=seed * 1000003 + a,
                                  polish_iters=200))
        res = anneal_batch(jobs, ctx=ctx)
        completed = attempts
        cands = [(r["rows"], r["L"]) for r in res if r["certified"]]
        converged = len(cands)
        # every candidate passes the gate again as the packing it would be written as
        if cands:
            checked = evaluate_batch([(n, c[0]) for c in cands], ctx=ctx)
            for (crows, _), (_, _, text, reason) in zip(cands, checked):
                if reason == "ok" and text is not None and float(text) < side:
                    rows, side = crows, float(text)
                    improvements += 1
    certify(n, rows, ctx=ctx)
    return rows, dict(n=n, seed=seed, attempts=completed, converged=converged, initial_L=start_side,
                      final_L=side, improvements=improvements)
