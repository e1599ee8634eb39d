"""The allocation-free certifier entry point (sqs_certify_batch_static).

Some callers cannot allocate GPU memory while they run: an application that
hands all device memory to its own pool up front, or a latency-critical loop
that forbids allocation after start-up.  For them the certifier has a form
whose scratch is one static device array.  Its verdicts must equal the
regular entry point's exactly, call after call, because the shared scratch
keeps the previous call's contents.

This file is collected last on purpose: it must pass on its own in a fresh
process and after every other test.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _call(fn_name, ctx, items, roundtrip=False):
    from sqs import _native as N
    from sqs.core import pack_batch
    n_of, row_start, sid, text, lit_off = pack_batch(items)
    out = (N.Verdict * len(items))()
    rc = getattr(N.lib(), fn_name)(ctx.handle, len(items), n_of.ctypes.data, row_start.ctypes.data,
                                   sid.ctypes.data, text, lit_off.ctypes.data, 1 if roundtrip else 0, out)
    N.check(rc)
    return [(v.ok, v.n, v.score, v.L.decode(), v.reason.decode()) for v in out]


def test_static_certifier_matches_regular_entry_point_on_two_calls(ctx):
    from sqs.workloads import certify_corpus
    cases = json.loads((GOLDEN / "certify_cases.json").read_text())
    first = [(c["n"], c["rows"]) for c in cases]
    second = certify_corpus(80, seed=23, n_hi=400, overlap_frac=0.2)
    # call 1: the golden cases; call 2: a different, larger batch with the
    # round-trip transform -- the second call must not see the first's state
    a1 = _call("sqs_certify_batch_static", ctx, first)
    a2 = _call("sqs_certify_batch_static", ctx, second, roundtrip=True)
    b1 = _call("sqs_certify_batch", ctx, first)
    b2 = _call("sqs_certify_batch", ctx, second, roundtrip=True)
    assert a1 == b1
    assert a2 == b2
    assert sum(v[0] for v in a1) > 0 and sum(not v[0] for v in a1) > 0
    # and once more in the other order, so a call following a larger one is covered
    assert _call("sqs_certify_batch_static", ctx, first) == b1


def test_static_certifier_rejects_oversized_calls(ctx):
    from sqs import SQSError
    from sqs.core import grid
    too_many_packings = [(1, grid(1))] * 4097
    with pytest.raises(SQSError):
        _call("sqs_certify_batch_static", ctx, too_many_packings)
    too_many_squares = [(1000, grid(1000))] * 17
    with pytest.raises(SQSError):
        _call("sqs_certify_batch_static", ctx, too_many_squares)
    # a rejected call leaves the entry point usable
    assert _call("sqs_certify_batch_static", ctx, [(4, grid(4))])[0][0] == 1
