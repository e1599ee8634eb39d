"""Serving: a continuous-batching request loop for anneal-and-certify jobs.

``Server`` wraps the native runtime (sqs_server_*): jobs are admitted by HBM
footprint while slots are free, run side by side in slices with their state
resident on the GPU, and are polished, certified and handed back as they
finish.  ``run_stream`` drives it with timed arrivals (for example Poisson)
and reports certified jobs/s with p50/p99 latency; ``run_plain`` runs the
same jobs one launch per job, the comparator.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _native as N
from .anneal import AnnealJob, _cjob, anneal_batch


def _result_dict(job: AnnealJob, r: N.JobResult, q: np.ndarray) -> dict:
    ok = bool(r.certified)
    return dict(n=job.n, status=int(r.status), certified=ok, L=r.L.decode() if ok else None,
                reason=r.reason.decode(), L_cert=float(r.L_cert), L_polished=float(r.L_polished),
                dilation=float(r.dilation), score=float(r.score), shrinks=int(r.shrinks),
                improvements=int(r.improvements), sweeps=int(r.sweeps_done), proposals=int(r.proposals),
                accepted=int(r.accepted), exchange_attempts=int(r.exchange_attempts),
                exchange_accepts=int(r.exchange_accepts), q=q.tolist() if ok else None)


class Server:
    """sqs_server: slice_sweeps sweeps of every admitted job per step, or,
    with slice_proposals, about that many proposals per replica of every job
    per step (its own sweep count, whole exchange intervals)."""

    def __init__(self, ctx: N.Context, hbm_bytes: int = 4 << 30, max_active: int = 512, slice_sweeps: int = 100,
                 *, slice_proposals: int | None = None):
        h = N._vp()
        slice_arg = -int(slice_proposals) if slice_proposals else slice_sweeps
        N.check(N.lib().sqs_server_create(ctx.handle, hbm_bytes, max_active, slice_arg, C.byref(h)))
        self.handle = h.value
        self.ctx = ctx
        self._jobs: dict[int, AnnealJob] = {}

    def close(self):
        if self.handle:
            N.lib().sqs_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, job: AnnealJob) -> int:
        cj = _cjob(job)
        jid = C.c_int64(0)
        N.check(N.lib().sqs_server_submit(self.handle, C.byref(cj), C.byref(jid)))
        self._jobs[jid.value] = job
        return jid.value

    def step(self) -> int:
        k = C.c_int(0)
        N.check(N.lib().sqs_server_step(self.handle, C.byref(k)))
        return k.value

    def poll(self, jid: int) -> dict | None:
        job = self._jobs.get(jid)  # unknown ids go to the library, which reports them
        r = N.JobResult()
        q = np.zeros((job.n if job else 1, 3))
        done = N.check(N.lib().sqs_server_poll(self.handle, jid, C.byref(r), q.ctypes.data_as(C.POINTER(C.c_double))))
        if not done:
            return None
        del self._jobs[jid]
        return _result_dict(job, r, q)

    def cancel(self, jid: int) -> None:
        N.check(N.lib().sqs_server_cancel(self.handle, jid))

    def info(self) -> tuple[int, int, int]:
        q, a, u = C.c_int(0), C.c_int(0), C.c_size_t(0)
        N.check(N.lib().sqs_server_info(self.handle, C.byref(q), C.byref(a), C.byref(u)))
        return q.value, a.value, u.value

    def stats(self) -> dict:
        """Steps, slice launches, jobs admitted and retired, host seconds per phase."""
        st = N.ServerStats()
        N.check(N.lib().sqs_server_get_stats(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in N.ServerStats._fields_}


def poisson_arrivals(count: int, rate: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def _latency_stats(lat: list[float], span: float, certified: int) -> dict:
    a = np.asarray(lat) if lat else np.zeros(1)
    return dict(jobs=len(lat), certified=certified, seconds=span,
                certified_jobs_per_s=certified / span if span > 0 else 0.0,
                p50_s=float(np.percentile(a, 50)), p99_s=float(np.percentile(a, 99)), mean_s=float(a.mean()))


def run_stream(server: Server, jobs: list[AnnealJob], arrivals, *, timeout: float = 600.0):
    """Submit job k at time arrivals[k] (seconds from the start) and step the
    server until every job is back.  Returns (results, stats)."""
    t0 = time.perf_counter()
    pending: dict[int, int] = {}
    results: list[dict | None] = [None] * len(jobs)
    done_at = [0.0] * len(jobs)
    k = 0
    while k < len(jobs) or pending:
        now = time.perf_counter() - t0
        if now > timeout:
            raise TimeoutError("stream did not drain in time")
        while k < len(jobs) and arrivals[k] <= now:
            pending[server.submit(jobs[k])] = k
            k += 1
        if not pending:
            time.sleep(max(0.0, arrivals[k] - now))
            continue
        server.step()
        now = time.perf_counter() - t0
        for jid in list(pending):
            r = server.poll(jid)
            if r is not None:
                idx = pending.pop(jid)
                results[idx] = r
                done_at[idx] = now
    lat = [done_at[i] - arrivals[i] for i in range(len(jobs))]
    span = max(done_at) - float(arrivals[0]) if jobs else 0.0
    return results, _latency_stats(lat, span, sum(bool(r and r["certified"]) for r in results))


def plain_service(ctx: N.Context, jobs: list[AnnealJob]) -> tuple[list[dict], list[float]]:
    """The comparator's service: every job alone in its own anneal, polish
    and certify launches.  Returns (results, seconds per job)."""
    results, service = [], []
    for job in jobs:
        t = time.perf_counter()
        results.append(anneal_batch([job], ctx=ctx)[0])
        service.append(time.perf_counter() - t)
    return results, service


def plain_stats(results: list[dict], service: list[float], arrivals) -> dict:
    """Latencies of the plain comparator serving jobs in arrival order (FIFO)
    with the given per-job service times."""
    finish, lat = 0.0, []
    for a, s in zip(arrivals, service):
        finish = max(finish, float(a)) + s
        lat.append(finish - float(a))
    span = finish - float(arrivals[0]) if len(service) else 0.0
    return _latency_stats(lat, span, sum(bool(r["certified"]) for r in results))


def run_plain_live(ctx: N.Context, jobs: list[AnnealJob], arrivals, *, timeout: float = 3600.0):
    """The comparator run live: jobs served one at a time in arrival order,
    each waiting for its arrival time, every job alone in its own anneal,
    polish and certify launches.  Returns (results, seconds per job, stats
    from the measured completion times)."""
    t0 = time.perf_counter()
    results, service, done_at = [], [], []
    for job, a in zip(jobs, arrivals):
        now = time.perf_counter() - t0
        if now > timeout:
            raise TimeoutError("plain stream did not drain in time")
        if now < a:
            time.sleep(a - now)
        t = time.perf_counter()
        results.append(anneal_batch([job], ctx=ctx)[0])
        service.append(time.perf_counter() - t)
        done_at.append(time.perf_counter() - t0)
    lat = [d - float(a) for d, a in zip(done_at, arrivals)]
    span = max(done_at) - float(arrivals[0]) if jobs else 0.0
    return results, service, _latency_stats(lat, span, sum(bool(r["certified"]) for r in results))


def run_plain(ctx: N.Context, jobs: list[AnnealJob], arrivals):
    """The comparator: every job alone in its own anneal/polish/certify
    launches, in arrival order (FIFO).  Returns (results, stats)."""
    results, service = plain_service(ctx, jobs)
    return results, plain_stats(results, service, arrivals)
