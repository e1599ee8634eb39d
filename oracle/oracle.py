"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracle.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
legs as the checker of the CUDA path.  The product never imports it.

``liboracle.so`` is this directory's own C/C++ restatement of the reference
algorithms.  ``_ref/`` holds the reference's own code compiled here (when its
sources were available at build time); ``ref_available()`` says whether it is.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_REF_SEEDED = None
_REF_CERT = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_cpp = C.POINTER(C.c_char_p)


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def lib():
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(str(path))
        L.sqo_pair.restype = C.c_double
        L.sqo_pair.argtypes = [_dp, _dp, _dp]
        L.sqo_pair_cached.restype = C.c_double
        L.sqo_pair_cached.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double, _dp, C.c_int]
        L.sqo_boundary.restype = C.c_double
        L.sqo_boundary.argtypes = [_dp, C.c_double, _dp]
        L.sqo_total.restype = C.c_double
        L.sqo_total.argtypes = [C.c_int, C.c_double, _dp, _dp, _i64p]
        L.sqo_total_smooth.restype = C.c_double
        L.sqo_total_smooth.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.sqo_total_batch.restype = C.c_int
        L.sqo_total_batch.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _i64p, C.c_int]
        L.sqo_certified_side.restype = C.c_double
        L.sqo_certified_side.argtypes = [C.c_int, _dp, _dp, _dp]
        L.sqo_certify.restype = C.c_int
        L.sqo_certify.argtypes = [C.c_int, C.c_int, _ip, _cpp, _cpp, _cpp, C.c_char_p, C.c_int,
                                  C.c_char_p, C.c_int, _dp]
        L.sqo_roundtrip.restype = None
        L.sqo_roundtrip.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.sqo_ptsa_batch.restype = C.c_int
        L.sqo_ptsa_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.sqo_certify_batch_text.restype = C.c_int
        L.sqo_certify_batch_text.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p,
                                             C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.sqo_certify_batch.restype = C.c_int
        L.sqo_certify_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p,
                                        C.c_int, C.c_void_p, C.c_void_p]
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return (HERE / "_ref" / "libref_seeded.so").exists() and (HERE / "_ref" / "libref_certifier.so").exists()


def ref_seeded():
    global _REF_SEEDED
    if _REF_SEEDED is None:
        L = C.CDLL(str(HERE / "_ref" / "libref_seeded.so"))
        L.ref_pair.restype = C.c_double
        L.ref_pair.argtypes = [_dp, _dp, _dp]
        L.ref_pair_smooth.restype = C.c_double
        L.ref_pair_smooth.argtypes = [_dp, _dp, _dp]
        L.ref_boundary.restype = C.c_double
        L.ref_boundary.argtypes = [_dp, C.c_double, _dp]
        L.ref_build_portfolio.restype = C.c_int
        L.ref_build_portfolio.argtypes = [C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp]
        L.ref_total_batch.restype = C.c_int
        L.ref_total_batch.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int]
        _REF_SEEDED = L
    return _REF_SEEDED


def ref_certifier():
    global _REF_CERT
    if _REF_CERT is None:
        L = C.CDLL(str(HERE / "_ref" / "libref_certifier.so"))
        L.ref_evaluate.restype = C.c_int
        L.ref_evaluate.argtypes = [C.c_int, C.c_int, _ip, _cpp, _cpp, _cpp, C.c_char_p, C.c_int,
                                   C.c_char_p, C.c_int, _dp]
        L.ref_roundtrip.restype = None
        L.ref_roundtrip.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.ref_evaluate_batch_text.restype = C.c_int
        L.ref_evaluate_batch_text.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p,
                                              C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_evaluate_batch.restype = C.c_int
        L.ref_evaluate_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p,
                                         C.c_int, C.c_void_p, C.c_void_p]
        _REF_CERT = L
    return _REF_CERT


# ---------------------------------------------------------------- energies
def pair(p, q, grad=False):
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    g = np.zeros(3) if grad else None
    e = lib().sqo_pair(_ptr(p, _dp), _ptr(q, _dp), _ptr(g, _dp))
    return (e, g) if grad else e


def total_batch(xya, L, grad=True, threads=None):
    """FP64 all-pairs energy (+ gradient, + candidate-pair counts) of a batch.

    xya: (configs, n, 3) float64; L: (configs,).  Returns (energy, grad, cand)."""
    xya = np.ascontiguousarray(xya, dtype=np.float64)
    configs, n, _ = xya.shape
    L = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (configs,)))
    e = np.zeros(configs)
    g = np.zeros_like(xya) if grad else None
    cand = np.zeros(configs, dtype=np.int64)
    threads = threads or os.cpu_count() or 1
    lib().sqo_total_batch(configs, n, _ptr(xya, _dp), _ptr(L, _dp), _ptr(e, _dp), _ptr(g, _dp),
                          _ptr(cand, _i64p), threads)
    return e, g, cand


def total_smooth(xya, L):
    """FP64 energy and smooth-variant gradient (the polish's) of one state."""
    xya = np.ascontiguousarray(xya, dtype=np.float64)
    g = np.zeros_like(xya)
    e = lib().sqo_total_smooth(xya.shape[0], float(L), _ptr(xya, _dp), _ptr(g, _dp))
    return e, g


def pair_cached(p, q, smooth=False):
    """sqo_pair_cached with cos/sin of the given angles: (energy, d/dp)."""
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    g = np.zeros(3)
    e = lib().sqo_pair_cached(_ptr(p, _dp), _ptr(q, _dp), np.cos(p[2]), np.sin(p[2]), np.cos(q[2]),
                              np.sin(q[2]), _ptr(g, _dp), 1 if smooth else 0)
    return e, g


def ref_total_batch(xya, L, grad=True, threads=None):
    """The reference's own pair()/boundary() all-pairs energy (+ gradient)."""
    xya = np.ascontiguousarray(xya, dtype=np.float64)
    configs, n, _ = xya.shape
    L = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (configs,)))
    e = np.zeros(configs)
    g = np.zeros_like(xya) if grad else None
    threads = threads or os.cpu_count() or 1
    used = ref_seeded().ref_total_batch(configs, n, _ptr(xya, _dp), _ptr(L, _dp), _ptr(e, _dp),
                                        _ptr(g, _dp), threads)
    return e, g, used


def ref_portfolio(n, L, seed_xya, chains, structured=1):
    """The reference's build_portfolio (seeded.cu:233-425): (chains, n, 3)."""
    seed = np.ascontiguousarray(seed_xya, dtype=np.float64)
    out = np.zeros((chains, n, 3))
    ref_seeded().ref_build_portfolio(n, chains, float(L), _ptr(seed, _dp), structured, _ptr(out, _dp))
    return out


def ref_portfolio_packing(n, L, seed_xya, chains):
    """The `packing` program's portfolio (dpack::build_portfolio): (chains, n, 3)."""
    lib_ = C.CDLL(str(HERE / "_ref" / "libref_packing.so"))
    lib_.ref_build_portfolio_packing.restype = C.c_int
    lib_.ref_build_portfolio_packing.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp]
    seed = np.ascontiguousarray(seed_xya, dtype=np.float64)
    out = np.zeros((chains, n, 3))
    lib_.ref_build_portfolio_packing(n, chains, float(L), _ptr(seed, _dp), _ptr(out, _dp))
    return out


def certified_side(xya):
    xya = np.ascontiguousarray(xya, dtype=np.float64)
    n = xya.shape[0]
    best = np.zeros_like(xya)
    lam = C.c_double(0)
    L = lib().sqo_certified_side(n, _ptr(xya, _dp), _ptr(best, _dp), C.byref(lam))
    return L, lam.value, best


class _Job(C.Structure):
    _fields_ = [("n", C.c_int), ("replicas", C.c_int), ("sweeps", C.c_int), ("exchange_every", C.c_int),
                ("L0", C.c_double), ("tmin", C.c_double), ("tmax", C.c_double), ("sigma_xy", C.c_double),
                ("sigma_a", C.c_double), ("shrink", C.c_double), ("seed", C.c_uint64), ("xya", _dp)]


class _JobOut(C.Structure):
    _fields_ = [("best_L", C.c_double), ("proposals", C.c_longlong), ("accepted", C.c_longlong),
                ("xatt", C.c_longlong), ("xacc", C.c_longlong), ("shrinks", C.c_int), ("pad", C.c_int)]


def ptsa_batch(jobs, threads=None):
    """CPU parallel tempering (sqo_ptsa_batch) of jobs given as objects with
    the fields of sqs.anneal.AnnealJob; returns (list of dicts, threads used)."""
    keep = [np.ascontiguousarray(j.xya, dtype=np.float64) for j in jobs]
    arr = (_Job * max(1, len(jobs)))()
    for k, (j, x) in enumerate(zip(jobs, keep)):
        arr[k] = _Job(x.shape[0], j.replicas, j.sweeps, j.exchange_every, j.L0, j.tmin, j.tmax, j.sigma_xy,
                      j.sigma_a, j.shrink, j.seed & 0xFFFFFFFFFFFFFFFF, x.ctypes.data_as(_dp))
    out = (_JobOut * max(1, len(jobs)))()
    used = lib().sqo_ptsa_batch(len(jobs), C.addressof(arr), C.addressof(out), threads or os.cpu_count() or 1)
    return [dict(best_L=o.best_L, proposals=o.proposals, accepted=o.accepted, exchange_attempts=o.xatt,
                 exchange_accepts=o.xacc, shrinks=o.shrinks) for o in out[:len(jobs)]], used


# ---------------------------------------------------------------- certifier
def _rows_to_c(rows):
    sid = np.array([int(r["square_id"]) for r in rows], dtype=np.int32)
    enc = [[str(r[k]).encode() for r in rows] for k in ("x", "y", "angle")]
    arrs = [(C.c_char_p * max(1, len(rows)))(*e) for e in enc]
    return sid, arrs


def certify(n, rows, which="oracle"):
    """(ok, L_or_None, reason, score) for one packing, by the oracle
    restatement (which="oracle") or the compiled reference ("ref")."""
    sid, (xs, ys, as_) = _rows_to_c(rows)
    Lbuf = C.create_string_buffer(128)
    rbuf = C.create_string_buffer(256)
    sc = C.c_double(0)
    fn = lib().sqo_certify if which == "oracle" else ref_certifier().ref_evaluate
    ok = fn(n, len(rows), _ptr(sid, _ip), xs, ys, as_, Lbuf, 128, rbuf, 256, C.byref(sc))
    return bool(ok), (Lbuf.value.decode() if ok else None), rbuf.value.decode(), sc.value


def roundtrip(s, which="oracle"):
    out = C.create_string_buffer(64)
    fn = lib().sqo_roundtrip if which == "oracle" else ref_certifier().ref_roundtrip
    fn(str(s).encode(), out, 64)
    return out.value.decode()


def certify_batch(n_of, row_start, sid, text, lit_off, which="oracle", threads=None):
    """Threaded batch certification of packed arrays (sqs.core.pack_batch
    layout): returns (ok int32[count], score float64[count], threads used)."""
    n_of = np.ascontiguousarray(n_of, np.int32)
    row_start = np.ascontiguousarray(row_start, np.int64)
    sid = np.ascontiguousarray(sid, np.int32)
    lit_off = np.ascontiguousarray(lit_off, np.int64)
    count = len(n_of)
    ok = np.zeros(count, np.int32)
    score = np.zeros(count)
    threads = threads or os.cpu_count() or 1
    fn = lib().sqo_certify_batch if which == "oracle" else ref_certifier().ref_evaluate_batch
    used = fn(count, n_of.ctypes.data, row_start.ctypes.data, sid.ctypes.data, text, lit_off.ctypes.data,
              threads, ok.ctypes.data, score.ctypes.data)
    return ok, score, used


def certify_batch_text(n_of, row_start, sid, text, lit_off, which="oracle", threads=None):
    """Threaded batch certification with the 50-decimal sides and reasons,
    by the oracle restatement (which="oracle") or the compiled reference
    ("ref"): (ok int32[count], score float64[count], L strings, reasons)."""
    n_of = np.ascontiguousarray(n_of, np.int32)
    row_start = np.ascontiguousarray(row_start, np.int64)
    sid = np.ascontiguousarray(sid, np.int32)
    lit_off = np.ascontiguousarray(lit_off, np.int64)
    count = len(n_of)
    ok = np.zeros(count, np.int32)
    score = np.zeros(count)
    Lb = C.create_string_buffer(80 * max(1, count))
    rb = C.create_string_buffer(112 * max(1, count))
    fn = lib().sqo_certify_batch_text if which == "oracle" else ref_certifier().ref_evaluate_batch_text
    fn(count, n_of.ctypes.data, row_start.ctypes.data, sid.ctypes.data, text, lit_off.ctypes.data,
       threads or os.cpu_count() or 1, ok.ctypes.data, score.ctypes.data, C.addressof(Lb), C.addressof(rb))
    raw_L, raw_r = Lb.raw, rb.raw
    Ls = [raw_L[80 * p:80 * (p + 1)].split(b"\0", 1)[0].decode() for p in range(count)]
    rs = [raw_r[112 * p:112 * (p + 1)].split(b"\0", 1)[0].decode() for p in range(count)]
    return ok, score, Ls, rs
