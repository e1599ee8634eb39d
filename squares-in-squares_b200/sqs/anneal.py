"""Anneal-and-certify jobs on the GPU: parallel-tempering annealing of n unit
squares in a shrinking container, FP64 best-state recompute, FP64 gradient
polish and interval certification of the best packing, batched.

A job's result depends only on its inputs and seed (counter-based RNG), so it
is the same whether the job runs alone, in a batch of other jobs, or sliced.
The result dictionaries carry the fields the reference's search programs
write into their raw JSON (seeded.cu:949-974, packing.cu:859-865) plus the
certified side.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

MAX_N = 1000


@dataclass
class AnnealJob:
    xya: np.ndarray                 # (n, 3) initial state: centre x, centre y, angle (radians)
    L0: float                       # initial container side
    replicas: int = 8
    sweeps: int = 1000              # one sweep = n proposals per replica; negative: -sweeps proposals
    exchange_every: int = 10        # sweeps between checkpoints; negative: -exchange_every proposals
    tmin: float = 1e-3
    tmax: float = 1e-1
    sigma_xy: float = 0.02
    sigma_a: float = 0.05
    shrink: float = 0.001
    seed: int = 42
    polish_iters: int = 200
    autotune: bool = False          # launch shape / cell side (and exchange_every=0) from the autotuner
    adapt: bool = False             # step adaptation, rung-scaled steps, cooling cycle (SQS_JOB_ADAPT)
    collective: bool = False        # row / column / disc / class / diagonal / tilted set moves (SQS_JOB_COLLECTIVE)
    kick: bool = False              # kick and reseed of overlapped replicas at exchange rounds (SQS_JOB_KICK)
    serial: bool = False            # one proposal at a time (SQS_JOB_SERIAL): same trajectory, for checking
    quench_all: bool = False        # quench every replica at exchange rounds (SQS_JOB_QUENCH_ALL)
    cert_all: bool = False          # dilation-certify every replica at checkpoints (SQS_JOB_CERT_ALL)
    quench_steps: int = 0           # 1..127: 16 k-iteration quenches without a slow-step exit (SQS_JOB_QUENCH_STEPS)
    targets: bool = False           # every rung in its own side below the best (SQS_JOB_TARGETS)
    ladders: int = 1                # rungs split into this many ladders (SQS_JOB_LADDERS)
    cluster: int = 0                # pinned cluster size (0: default / tuned)
    cell_index: int = 0             # pinned cell side index (0: 1.59, 1: 1.75, 2: 1.95, 3: 2.2)
    xya_rep: np.ndarray | None = None  # (replicas, n, 3) per-replica starts, e.g. from portfolio()
    n: int = field(init=False)

    def __post_init__(self):
        self.xya = np.ascontiguousarray(self.xya, dtype=np.float64).reshape(-1, 3)
        self.n = self.xya.shape[0]
        if not 0 <= self.quench_steps <= 127:
            raise ValueError("quench_steps must be in 0..127")
        if not 1 <= self.ladders <= 15:
            raise ValueError("ladders must be in 1..15")
        if self.xya_rep is not None:
            self.xya_rep = np.ascontiguousarray(self.xya_rep, dtype=np.float64).reshape(self.replicas, self.n, 3)


def _flags(j: AnnealJob) -> int:
    return ((N.JOB_AUTOTUNE if j.autotune else 0) | (N.JOB_ADAPT if j.adapt else 0) |
            (N.JOB_COLLECTIVE if j.collective else 0) | (N.JOB_KICK if j.kick else 0) |
            (N.JOB_SERIAL if j.serial else 0) | (N.JOB_QUENCH_ALL if j.quench_all else 0) |
            (N.JOB_CERT_ALL if j.cert_all else 0) | (N.JOB_TARGETS if j.targets else 0) |
            ((j.ladders if j.ladders > 1 else 0) << 20) | (j.quench_steps << 24) |
            (j.cluster << 8) | (j.cell_index << 16))


def _cjob(j: AnnealJob) -> N.Job:
    return N.Job(n=j.n, replicas=j.replicas, sweeps=j.sweeps, exchange_every=j.exchange_every,
                 polish_iters=j.polish_iters, flags=_flags(j), L0=j.L0, tmin=j.tmin, tmax=j.tmax, sigma_xy=j.sigma_xy,
                 sigma_a=j.sigma_a, shrink=j.shrink, seed=j.seed & 0xFFFFFFFFFFFFFFFF,
                 xya=j.xya.ctypes.data_as(C.POINTER(C.c_double)),
                 xya_rep=j.xya_rep.ctypes.data_as(C.POINTER(C.c_double)) if j.xya_rep is not None else None)


def _trace_buffers(j: AnnealJob) -> dict:
    R, n = j.replicas, j.n
    return dict(xya=np.zeros((R, n, 3), np.float32), energy=np.zeros(R), energy_full=np.zeros(R),
                L_cert=np.zeros(R), dilation=np.zeros(R), side=np.zeros(R, np.float32),
                temperature=np.zeros(R, np.float32), step_scale=np.zeros(R, np.float32),
                rung=np.zeros(R, np.int32))


def _ctrace(b: dict) -> N.ReplicaTrace:
    t = N.ReplicaTrace()
    for name, arr in b.items():
        ct = {np.dtype(np.float32): C.c_float, np.dtype(np.float64): C.c_double,
              np.dtype(np.int32): C.c_int32}[arr.dtype]
        setattr(t, name, arr.ctypes.data_as(C.POINTER(ct)))
    return t


def anneal_batch(jobs: list[AnnealJob], *, ctx: N.Context | None = None, slice_sweeps: int = 0,
                 trace: bool = False) -> list[dict]:
    """Run jobs in batched launches; returns one result dict per job.  With
    trace=True (sqs_anneal_batch_trace) each dict also has "trace": every
    replica's final FP32 state, its running and recomputed energies, its FP64
    certified side, side, temperature, step scale and rung."""
    own = ctx is None
    ctx = ctx or N.Context(0)
    tbufs = [_trace_buffers(j) for j in jobs] if trace else None
    tstructs = (N.ReplicaTrace * max(1, len(jobs)))(*[_ctrace(b) for b in tbufs]) if trace else None
    try:
        arr = (N.Job * max(1, len(jobs)))(*[_cjob(j) for j in jobs])
        res = (N.JobResult * max(1, len(jobs)))()
        outs = [np.zeros((j.n, 3)) for j in jobs]
        ptrs = (C.POINTER(C.c_double) * max(1, len(jobs)))(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
        if trace:
            N.check(N.lib().sqs_anneal_batch_trace(ctx.handle, arr, len(jobs), slice_sweeps, ptrs, res, tstructs))
        else:
            N.check(N.lib().sqs_anneal_batch(ctx.handle, arr, len(jobs), slice_sweeps, ptrs, res))
    finally:
        if own:
            ctx.close()
    out = []
    for k, (j, r, q) in enumerate(zip(jobs, res, outs)):
        ok = bool(r.certified)
        rows = [dict(square_id=str(i), x=format(float(x), ".17g"), y=format(float(y), ".17g"),
                     angle=format(float(a), ".17g")) for i, (x, y, a) in enumerate(q)] if ok else None
        out.append(dict(
            n=j.n, status=int(r.status), certified=ok, L=r.L.decode() if ok else None,
            reason=r.reason.decode(), target_L=float(r.L_cert), L_cert=float(r.L_cert),
            L_polished=float(r.L_polished), dilation=float(r.dilation), score=float(r.score),
            shrinks=int(r.shrinks), improvements=int(r.improvements), sweeps=int(r.sweeps_done),
            chains=int(r.replicas), proposals=int(r.proposals), accepted=int(r.accepted),
            exchange_attempts=int(r.exchange_attempts), exchange_accepts=int(r.exchange_accepts),
            device_ms=float(r.device_ms), q=q.tolist() if ok else None, rows=rows,
            launch=dict(cluster_ctas=int(r.cluster_ctas), replicas_per_cta=int(r.replicas_per_cta),
                        exchange_every=int(r.exchange_every), cell_side=float(r.cell_side),
                        overflows=int(r.overflows))))
        if trace:
            t = dict(tbufs[k])
            t["exchange_rounds"] = int(tstructs[k].exchange_rounds)
            t["cells_ok"] = bool(tstructs[k].cells_ok)
            out[-1]["trace"] = t
    return out


def autotune(job: AnnealJob, *, ctx: N.Context | None = None, latency: bool = False) -> dict:
    """The autotuner's launch shape for a job's class (sqs_autotune)."""
    own = ctx is None
    ctx = ctx or N.Context(0)
    try:
        t = N.Tuning()
        cj = _cjob(job)
        N.check(N.lib().sqs_autotune(ctx.handle, C.byref(cj), N.TUNE_LATENCY if latency else 0, C.byref(t)))
    finally:
        if own:
            ctx.close()
    return dict(cluster_ctas=t.cluster_ctas, replicas_per_cta=t.replicas_per_cta, exchange_every=t.exchange_every,
                trials=t.trials, cell_side=t.cell_side, us_per_sweep=t.us_per_sweep)


def jittered_grid(n: int, jitter: float = 0.05, angle_hi: float = 0.1, seed: int = 42):
    """Grid centres at half-integers (ceil(sqrt n) columns) plus uniform jitter
    and small angles: the plain single-instance configuration's start."""
    rng = np.random.default_rng(seed)
    w = math.isqrt(n - 1) + 1
    i = np.arange(n)
    xy = np.stack([i % w + 0.5, i // w + 0.5], axis=1) + rng.uniform(-jitter, jitter, (n, 2))
    return np.concatenate([xy, rng.uniform(0.0, angle_hi, (n, 1))], axis=1), float(w)


def portfolio(seed_xya, L: float, chains: int, *, structured: bool = True, seed: int = 0,
              jitter: bool = True) -> np.ndarray:
    """Initial states of `chains` search chains, (chains, n, 3): the
    reference's structured portfolio (sqs_portfolio; seeded.cu:233-451).
    Chains 8k .. 8k + 7 are the replicas of the k-th 8-replica job."""
    seed_xya = np.ascontiguousarray(seed_xya, dtype=np.float64).reshape(-1, 3)
    n = seed_xya.shape[0]
    out = np.zeros((chains, n, 3))
    N.check(N.lib().sqs_portfolio(n, float(L), seed_xya.ctypes.data_as(C.POINTER(C.c_double)), chains,
                                  int(structured), seed & 0xFFFFFFFFFFFFFFFF, int(jitter),
                                  out.ctypes.data_as(C.POINTER(C.c_double))))
    return out
