"""The allocation-free certifier entry point (sqs_certify_batch_static).

Some callers cannot allocate GPU memory while they run: an application that
hands all device memory to its own pool up front, or a latency-critical loop
that forbids allocation after start-up.  For them the certifier has a form
whose scratch is one static device array.  Its verdicts must equal the
regular entry point's exactly, call after call, because the shared scratch
keeps the previous call's contents.

The first call on a device (a call with count = 0 does only this) sets the
path up: it loads the module and kernels and lets the driver size their
local memory.  After it, calls must leave the device's free memory and the
context's staging buffers exactly as they were.

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


def _deep_cases():
    # two squares whose separation is decided only past 63 digits (the 15-
    # and 58-limb stages of the per-pair kernel), both signs
    from test_certify_gpu import _deep_pair
    items = []
    for theta in ("0.5", "1.1", "0.25", "1.5"):
        for k in (70, 80, 90, 120):
            for sign in (1, -1):
                items.append((2, _deep_pair(theta, k, sign)))
    return items


def test_static_certifier_deep_stages_match_regular_entry_point(ctx):
    deep = _deep_cases()
    a = _call("sqs_certify_batch_static", ctx, deep)
    b = _call("sqs_certify_batch", ctx, deep)
    assert a == b
    reasons = {v[4] for v in a}
    assert "ok" in reasons and "infeasible: Squares overlap (certified)" in reasons
    assert _call("sqs_certify_batch_static", ctx, deep) == b


def test_static_certifier_allocates_nothing_after_set_up():
    import json as _json

    from sqs import Context
    from sqs.workloads import certify_corpus
    cases = _json.loads((GOLDEN / "certify_cases.json").read_text())
    batches = [[(c["n"], c["rows"]) for c in cases], _deep_cases(), certify_corpus(60, seed=31, n_hi=300)]
    with Context(0) as c:
        # set-up call: count = 0
        assert _call("sqs_certify_batch_static", c, []) == []
        m0 = c.memory()
        assert m0["staging_device"] == 0 and m0["staging_host"] == 0
        for _ in range(2):
            for items in batches:
                _call("sqs_certify_batch_static", c, items)
            _call("sqs_certify_batch_static", c, batches[2], roundtrip=True)
        m1 = c.memory()
        assert m1["device_free"] == m0["device_free"], (m0, m1)
        assert m1["staging_device"] == 0 and m1["staging_host"] == 0, m1


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
