"""ctypes binding of libsqs.so (the C ABI declared in include/sqs.h).

There is no fallback: if the library is missing or no sm_100 device is
visible, the calls raise.  No PyTorch is involved; arrays are numpy.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libsqs.so"

_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_cpp = C.POINTER(C.c_char_p)


class SQSError(RuntimeError):
    """A libsqs call returned a negative status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libsqs error {code}: {message}")
        self.code = code


class Verdict(C.Structure):
    """sqs_verdict (include/sqs.h)."""
    _fields_ = [("ok", C.c_int32), ("n", C.c_int32), ("score", C.c_double),
                ("L", C.c_char * 80), ("reason", C.c_char * 112)]


class Job(C.Structure):
    """sqs_job (include/sqs.h)."""
    _fields_ = [("n", C.c_int32), ("replicas", C.c_int32), ("sweeps", C.c_int32), ("exchange_every", C.c_int32),
                ("polish_iters", C.c_int32), ("flags", C.c_int32), ("L0", C.c_double), ("tmin", C.c_double),
                ("tmax", C.c_double), ("sigma_xy", C.c_double), ("sigma_a", C.c_double), ("shrink", C.c_double),
                ("seed", C.c_uint64), ("xya", C.POINTER(C.c_double)), ("xya_rep", C.POINTER(C.c_double))]


class JobResult(C.Structure):
    """sqs_job_result (include/sqs.h)."""
    _fields_ = [("status", C.c_int32), ("certified", C.c_int32), ("shrinks", C.c_int32),
                ("improvements", C.c_int32), ("sweeps_done", C.c_int32), ("replicas", C.c_int32),
                ("cluster_ctas", C.c_int32), ("replicas_per_cta", C.c_int32), ("exchange_every", C.c_int32),
                ("overflows", C.c_int32), ("cell_side", C.c_double),
                ("L_cert", C.c_double), ("L_polished", C.c_double), ("dilation", C.c_double),
                ("score", C.c_double), ("proposals", C.c_int64), ("accepted", C.c_int64),
                ("exchange_attempts", C.c_int64), ("exchange_accepts", C.c_int64), ("device_ms", C.c_double),
                ("L", C.c_char * 80), ("reason", C.c_char * 112)]


class ReplicaTrace(C.Structure):
    """sqs_replica_trace (include/sqs.h)."""
    _fields_ = [("xya", C.POINTER(C.c_float)), ("energy", C.POINTER(C.c_double)),
                ("energy_full", C.POINTER(C.c_double)), ("L_cert", C.POINTER(C.c_double)),
                ("dilation", C.POINTER(C.c_double)), ("side", C.POINTER(C.c_float)),
                ("temperature", C.POINTER(C.c_float)), ("step_scale", C.POINTER(C.c_float)),
                ("rung", C.POINTER(C.c_int32)), ("exchange_rounds", C.c_int32), ("cells_ok", C.c_int32)]


class Tuning(C.Structure):
    """sqs_tuning (include/sqs.h)."""
    _fields_ = [("cluster_ctas", C.c_int32), ("replicas_per_cta", C.c_int32), ("exchange_every", C.c_int32),
                ("trials", C.c_int32), ("cell_side", C.c_double), ("us_per_sweep", C.c_double)]


class PolishResult(C.Structure):
    """sqs_polish_result (include/sqs.h)."""
    _fields_ = [("L_in", C.c_double), ("L_out", C.c_double), ("iterations", C.c_int32), ("improved", C.c_int32)]


class ServerStats(C.Structure):
    """sqs_server_stats (include/sqs.h)."""
    _fields_ = [("steps", C.c_int64), ("slices", C.c_int64), ("admitted", C.c_int64), ("retired", C.c_int64),
                ("admit_s", C.c_double), ("launch_s", C.c_double), ("retire_s", C.c_double), ("wait_s", C.c_double),
                ("polish_s", C.c_double), ("certify_s", C.c_double)]


JOB_AUTOTUNE = 1
JOB_ADAPT = 2
JOB_COLLECTIVE = 4
JOB_KICK = 8
JOB_SERIAL = 16
JOB_QUENCH_ALL = 32
JOB_CERT_ALL = 64
JOB_TARGETS = 128
TUNE_LATENCY = 1


# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "sqs_version": (C.c_char_p, []),
    "sqs_last_error": (C.c_char_p, []),
    "sqs_device_count": (C.c_int, []),
    "sqs_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "sqs_ctx_destroy": (C.c_int, [_vp]),
    "sqs_ctx_device_info": (C.c_int, [_vp, C.c_char_p, C.c_int, _ip]),
    "sqs_dev_alloc": (C.c_int, [_vp, C.c_size_t, C.POINTER(_vp)]),
    "sqs_dev_free": (C.c_int, [_vp, _vp]),
    "sqs_copy_h2d": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "sqs_copy_d2h": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "sqs_memset": (C.c_int, [_vp, _vp, C.c_int, C.c_size_t]),
    "sqs_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_vp)]),
    "sqs_host_free": (C.c_int, [_vp]),
    "sqs_sync": (C.c_int, [_vp]),
    "sqs_event_record": (C.c_int, [_vp, C.c_int]),
    "sqs_event_elapsed": (C.c_int, [_vp, C.c_int, C.c_int, _fp]),
    "sqs_flush_l2": (C.c_int, [_vp]),
    "sqs_ctx_memory": (C.c_int, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                 C.POINTER(C.c_size_t)]),
    "sqs_launch_count": (C.c_int64, [_vp]),
    "sqs_graph_replay_count": (C.c_int64, [_vp]),
    "sqs_sat_energy": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int]),
    "sqs_sat_energy_host": (C.c_int, [_vp, C.c_int, C.c_int, _fp, _fp, _fp, _fp, _u32p]),
    "sqs_certify_batch": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_char_p, _vp, C.c_int, C.POINTER(Verdict)]),
    "sqs_certify_batch_static": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_char_p, _vp, C.c_int,
                                           C.POINTER(Verdict)]),
    "sqs_anneal_batch": (C.c_int, [_vp, C.POINTER(Job), C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_double)),
                                   C.POINTER(JobResult)]),
    "sqs_anneal_batch_trace": (C.c_int, [_vp, C.POINTER(Job), C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_double)),
                                         C.POINTER(JobResult), C.POINTER(ReplicaTrace)]),
    "sqs_energy_fp64": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sqs_server_create": (C.c_int, [_vp, C.c_size_t, C.c_int, C.c_int, C.POINTER(_vp)]),
    "sqs_server_destroy": (C.c_int, [_vp]),
    "sqs_server_submit": (C.c_int, [_vp, C.POINTER(Job), C.POINTER(C.c_int64)]),
    "sqs_server_step": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "sqs_server_poll": (C.c_int, [_vp, C.c_int64, C.POINTER(JobResult), C.POINTER(C.c_double)]),
    "sqs_server_cancel": (C.c_int, [_vp, C.c_int64]),
    "sqs_portfolio": (C.c_int, [C.c_int, C.c_double, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_uint64, C.c_int,
                                C.POINTER(C.c_double)]),
    "sqs_polish_batch": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int,
                                   C.POINTER(C.c_double), C.POINTER(PolishResult)]),
    "sqs_autotune": (C.c_int, [_vp, C.POINTER(Job), C.c_int, C.POINTER(Tuning)]),
    "sqs_server_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "sqs_server_get_stats": (C.c_int, [_vp, C.POINTER(ServerStats)]),
}

_LIB = None


def lib():
    """Load libsqs.so once (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing; build it with "
                               "`python squares-in-squares_b200/build.py`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int) -> int:
    if rc < 0:
        raise SQSError(rc, lib().sqs_last_error().decode(errors="replace"))
    return rc


def ptr(a: np.ndarray | None, t=_vp):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to libsqs must be C-contiguous"
    return a.ctypes.data_as(t)


class DeviceArray:
    """A device buffer owned by a Context (numpy-like shape/dtype metadata)."""

    def __init__(self, ctx: "Context", shape, dtype):
        self.ctx = ctx
        self.shape = tuple(int(s) for s in np.atleast_1d(shape))
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = _vp()
        check(lib().sqs_dev_alloc(ctx.handle, max(1, self.nbytes), C.byref(p)))
        self.ptr = p.value

    def upload(self, host: np.ndarray):
        host = np.ascontiguousarray(host, dtype=self.dtype)
        assert host.nbytes == self.nbytes
        check(lib().sqs_copy_h2d(self.ctx.handle, self.ptr, host.ctypes.data, self.nbytes))
        return self

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self.shape, self.dtype) if out is None else out
        check(lib().sqs_copy_d2h(self.ctx.handle, out.ctypes.data, self.ptr, self.nbytes))
        self.ctx.sync()
        return out

    def free(self):
        if self.ptr:
            check(lib().sqs_dev_free(self.ctx.handle, self.ptr))
            self.ptr = None


class PinnedArray:
    """Page-locked host array (numpy view) for timed transfers."""

    def __init__(self, shape, dtype):
        self.dtype = np.dtype(dtype)
        self.shape = tuple(int(s) for s in np.atleast_1d(shape))
        nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = _vp()
        check(lib().sqs_host_alloc(max(1, nbytes), C.byref(p)))
        self._p = p.value
        buf = (C.c_char * max(1, nbytes)).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(self.shape))).reshape(self.shape)

    def free(self):
        if self._p:
            self.array = None
            check(lib().sqs_host_free(self._p))
            self._p = None


class Context:
    """One CUDA device + stream (sqs_ctx)."""

    def __init__(self, device: int = 0):
        h = _vp()
        check(lib().sqs_ctx_create(device, C.byref(h)))
        self.handle = h.value
        self.device = device

    def close(self):
        if self.handle:
            lib().sqs_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self):
        buf = C.create_string_buffer(256)
        sm = C.c_int(0)
        check(lib().sqs_ctx_device_info(self.handle, buf, 256, C.byref(sm)))
        return buf.value.decode(), sm.value

    def sync(self):
        check(lib().sqs_sync(self.handle))

    def record(self, slot: int):
        check(lib().sqs_event_record(self.handle, slot))

    def elapsed(self, a: int, b: int) -> float:
        ms = C.c_float(0)
        check(lib().sqs_event_elapsed(self.handle, a, b, C.byref(ms)))
        return ms.value

    def flush_l2(self):
        check(lib().sqs_flush_l2(self.handle))

    def launches(self) -> int:
        return int(lib().sqs_launch_count(self.handle))

    def memory(self) -> dict:
        """Device memory free / total and the bytes the context's own staging
        buffers hold on the device and in pinned host memory."""
        v = [C.c_size_t(0) for _ in range(4)]
        check(lib().sqs_ctx_memory(self.handle, *[C.byref(x) for x in v]))
        return dict(device_free=v[0].value, device_total=v[1].value, staging_device=v[2].value,
                    staging_host=v[3].value)

    def graph_replays(self) -> int:
        return int(lib().sqs_graph_replay_count(self.handle))

    def alloc(self, shape, dtype) -> DeviceArray:
        return DeviceArray(self, shape, dtype)


def device_count() -> int:
    return int(lib().sqs_device_count())
