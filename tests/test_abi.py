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
