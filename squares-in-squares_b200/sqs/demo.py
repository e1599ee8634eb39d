"""The raw-search-output gate of the reference's cuda/demo.py:
``certified_candidate(raw)`` (demo.py:25-40) dilates the centres of a search
program's best state by 1.000002, 1.00001, 1.0001 in turn and returns the
first packing the official certifier accepts, as (rows, L, dilation); it
raises ValueError otherwise.  All three rungs are certified in one GPU
batch here."""
from __future__ import annotations

import numpy as np

from . import _native as N
from .polish import ladder_certify

CANDIDATE_LADDER = (1.000002, 1.00001, 1.0001)


def certified_candidate(raw: dict, *, ctx: N.Context | None = None):
    n = raw["n"]
    q = np.asarray(raw["q"], dtype=np.float64)
    if q.shape != (n, 3) or not np.isfinite(q).all():
        raise ValueError("no finite GPU zero-energy candidate")
    got = ladder_certify([q], CANDIDATE_LADDER, ctx=ctx)[0]
    if got is None:
        raise ValueError("official certifier rejected GPU candidate")
    return got
