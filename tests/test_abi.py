"""The C ABI: the library loads, exports every entry point include/sqs.h
declares, and reports errors through status codes + sqs_last_error()."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(sqs_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from sqs import _native as N
    lib = ctypes.CDLL(str(N.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes table covers the whole header, with no stale names
    assert set(N.SIGNATURES) == names


def test_version_and_error_reporting_without_gpu():
    from sqs import _native as N
    L = N.lib()
    assert b"sm_100a" in L.sqs_version()
    if N.device_count() == 0:
        with pytest.raises(N.SQSError) as e:
            N.Context(0)
        assert e.value.code == -1
        assert "not present" in str(e.value)


def test_job_flag_constants_match_the_header():
    from sqs import _native as N
    text = (ROOT / "include" / "sqs.h").read_text()
    defs = dict(re.findall(r"#define SQS_(JOB_[A-Z_]+) (\d+)\b", text))
    assert {"JOB_AUTOTUNE", "JOB_SERIAL", "JOB_QUENCH_ALL", "JOB_CERT_ALL"} <= set(defs)
    for name, value in defs.items():
        assert getattr(N, name) == int(value), name
    # the packed fields sit above the single-bit options and below the sign bit
    assert "#define SQS_JOB_QUENCH_STEPS(k) ((int32_t)(k) << 24)" in text


def test_anneal_job_checks_the_quench_budget():
    import numpy as np

    from sqs.anneal import AnnealJob, _flags
    xya = np.zeros((4, 3))
    assert _flags(AnnealJob(xya, L0=2.0, quench_steps=127, cert_all=True)) == (127 << 24) | 64
    with pytest.raises(ValueError):
        AnnealJob(xya, L0=2.0, quench_steps=128)
