#!/usr/bin/env python
"""Benchmark of the hot path; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sqs|reference]

Workload (N=1): the SAT overlap-energy microbench -- 4,096 independent
configurations of n=200 unit squares, centres uniform in [0, L]^2 with
L = 1.05 sqrt(200), angles uniform in [0, pi/2) (seeded synthetic data),
FP32 cell-list energy + gradient.  A step is one launch over all 4,096
configurations; the metric is SAT pair-tests/s, counting candidate pairs
(centre distance^2 < 2) evaluated per second.  L2 is flushed (256 MiB
memset) before every timed launch; each launch is timed with CUDA events on
the launching stream.

Under torchrun (N > 1) every rank runs the same workload on its own GPU
(replicas: the path has no exchange step), timing is the max over ranks and
`value` the sum of all ranks' pair tests over that time (weak scaling).

--impl reference times the reference's own CPU implementation of the path
(its FP64 pair()/boundary() from seeded.cu, compiled into oracle/_ref; the
oracle restatement when _ref is absent) on all host cores, same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "squares-in-squares_b200"))

METRIC = "SAT pair-tests/s"
UNIT = "pair-tests/s"
CONFIGS, NSQ, SEED = 4096, 200, 42
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------ plumbing
class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.pg = None
        if self.world > 1:
            from datetime import timedelta

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [s for s in cvd.split(",") if s.strip()]
        self.sel = ids[local_rank] if local_rank < len(ids) else str(local_rank)
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"sqs_clocks_{os.getpid()}_{local_rank}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", self.sel, "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for name, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons),
                    samples=len(sm))


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_metric(kernel: str, key: str) -> float | None:
    """A figure of `kernel` from the committed ncu summary (profiles/traffic.json)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())[kernel][key])
    except (KeyError, ValueError, TypeError):
        return None


def ncu_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())[kernel]["dram_bytes_per_launch"])
    except (KeyError, ValueError, TypeError):
        return None


# ------------------------------------------------------------------ workload
def workload():
    import numpy as np

    from sqs.workloads import sat_microbench

    xya, side = sat_microbench(CONFIGS, NSQ, SEED)
    return xya.astype(np.float32), side.astype(np.float32)


def algorithmic_bytes(configs: int, n: int) -> int:
    # in: 12 B/square + 4 B side; out: 12 B/square gradient + 4 B energy + 4 B count
    return configs * (n * 24 + 12)


def cpu_pairs_per_s(x32, s32, seconds: float, configs_per_step: int | None = None, steps: int | None = None,
                    warmup: int = 0):
    """Time the reference's CPU path (oracle/_ref if built, else the oracle
    port) on all host cores.  Returns (value, kind, cores, sample, n_steps, sec)."""
    import numpy as np

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    x64 = x32.astype(np.float64)
    s64 = s32.astype(np.float64)
    _, _, cand = O.total_batch(x64, s64, grad=False, threads=threads)
    kind = "reference" if O.ref_available() else "port"
    run = (lambda a, b: O.ref_total_batch(a, b, grad=True, threads=threads)) if kind == "reference" else \
        (lambda a, b: O.total_batch(a, b, grad=True, threads=threads))
    per = configs_per_step or x64.shape[0]
    for w in range(warmup):
        i = (w * per) % x64.shape[0]
        run(x64[i:i + per], s64[i:i + per])
    done_pairs, t0, k = 0, time.perf_counter(), 0
    while True:
        i = (k * per) % x64.shape[0]
        run(x64[i:i + per], s64[i:i + per])
        done_pairs += int(cand[i:i + per].sum())
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (steps is None and el >= seconds):
            break
    sample = (f"{k} passes of {per} of the {x64.shape[0]} n={x64.shape[1]} configurations, "
              f"FP64 all-pairs energy + gradient, {threads} threads")
    return done_pairs / el, kind, threads, sample, k, el


def accuracy(d_e, d_g, x32, s32, configs: int = 64) -> dict:
    """FP32 energies and gradients of the last launch against the FP64
    all-pairs energy of the same FP32 inputs (the oracle restatement of
    seeded.cu:92-162) on the first `configs` configurations."""
    import numpy as np

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    e = d_e.download()[:configs].astype(np.float64)
    g = d_g.download()[:configs].astype(np.float64)
    eo, go, _ = O.total_batch(x32[:configs].astype(np.float64), s32[:configs].astype(np.float64))
    rel = np.abs(e - eo) / np.maximum(np.abs(eo), 1e-30)
    return dict(configs=configs, max_rel_energy_error=float(rel.max()), mean_rel_energy_error=float(rel.mean()),
                max_abs_grad_error=float(np.abs(g - go).max()), vs="FP64 all-pairs oracle on the same FP32 inputs")


def anneal_accuracy(ctx) -> dict:
    """FP32 annealer energies against the FP64 oracle, per configuration.

    Every replica's final FP32 state is read back with the annealer's running
    fixed-point energy (sqs_anneal_batch_trace); the oracle's FP64 all-pairs
    total of the same state and side is the reference.  Reports, per
    configuration, the largest relative and absolute error and whether every
    running energy equals its from-scratch recompute bit for bit."""
    import numpy as np

    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle as O

    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid

    def plain():
        xya, L0 = jittered_grid(10, seed=42)
        return [AnnealJob(xya, L0=L0, replicas=8, sweeps=20000, exchange_every=10, tmin=1e-3, tmax=1e-1, seed=42,
                          polish_iters=0)]

    def batched():
        rng = np.random.default_rng(42)
        out = []
        for k in range(32):
            n = int(rng.integers(20, 401))
            xya, L0 = jittered_grid(n, seed=k)
            out.append(AnnealJob(xya, L0=L0, replicas=32, sweeps=200, exchange_every=10, tmin=1e-4, tmax=5e-2,
                                 seed=k, polish_iters=0))
        return out

    def served():
        out = []
        for k, job in enumerate(served_jobs(12, sweeps=100)):
            job.polish_iters = 0
            out.append(job)
        return out

    res = {}
    for name, make, what in (("plain_pt", plain, "n=10, 8 replicas, 20,000 sweeps (all replicas)"),
                             ("batched", batched, "32 of the batched instances (n U[20,400], 32 replicas), "
                                                  "200 sweeps"),
                             ("served", served, "12 jobs of the served stream (n log-uniform [5,1000], "
                                                "16-64 replicas), 100 sweeps")):
        jobs = make()
        out = anneal_batch(jobs, ctx=ctx, trace=True)
        rel, ab, exact, reps = 0.0, 0.0, True, 0
        for r in out:
            t = r["trace"]
            eo, _, _ = O.total_batch(t["xya"].astype(np.float64), t["side"].astype(np.float64), grad=False)
            d = np.abs(t["energy"] - eo)
            ab = max(ab, float(d.max()))
            rel = max(rel, float((d / np.maximum(eo, 1e-30)).max()))
            exact &= bool(np.array_equal(t["energy"], t["energy_full"]))
            reps += len(d)
        res[name] = dict(workload=what, replicas=reps, max_rel_energy_error=rel, max_abs_energy_error=ab,
                         running_equals_recompute=exact,
                         tolerance="1e-5 relative, 1e-5 absolute floor (reference globaltest.cu:49)")
    res["vs"] = "FP64 all-pairs oracle on the same FP32 states and sides"
    return res


def run_reference(args, D: Dist):
    if D.rank != 0:
        return
    x32, s32 = workload()
    per = 256
    val, kind, cores, sample, k, el = cpu_pairs_per_s(x32, s32, 0, configs_per_step=per, steps=args.steps,
                                                      warmup=args.warmup)
    line = dict(metric=METRIC, value=val, unit=UNIT, impl="reference", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=1e3 * el / max(k, 1), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic",
                config=dict(workload=f"SAT energy+gradient, {CONFIGS} configs x n={NSQ}, "
                                     f"{per} configs per step", configs=CONFIGS, n=NSQ, seed=SEED),
                cpu_baseline=dict(value=val, unit=UNIT, cores=cores, kind=kind, sample=sample),
                e2e=dict(value=val, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def run_sqs(args, D: Dist):
    import numpy as np

    from sqs import Context, _native as N, sat

    x32, s32 = workload()
    configs, n, _ = x32.shape
    ctx = Context(D.local)
    name, sms = ctx.info()
    d_x = ctx.alloc(x32.shape, np.float32).upload(x32)
    d_s = ctx.alloc((configs,), np.float32).upload(s32)
    d_e = ctx.alloc((configs,), np.float32)
    d_g = ctx.alloc(x32.shape, np.float32)
    d_c = ctx.alloc((configs,), np.uint32)
    threads = args.threads
    # candidate pairs per launch (numerator of the metric), from the kernel's own count
    sat.energy_device(ctx, configs, n, d_x, d_s, d_e, d_g, d_c, threads=threads)
    pairs_per_step = int(d_c.download().sum())
    for _ in range(max(3, args.warmup)):
        ctx.flush_l2()
        sat.energy_device(ctx, configs, n, d_x, d_s, d_e, d_g, None, threads=threads)
    ctx.sync()
    D.barrier()
    clocks = Clocks(D.local)
    clocks.start()
    time.sleep(0.15)
    launches0 = ctx.launches()
    kernel_ms = []
    K = args.steps
    done = 0
    while done < K:
        chunk = min(32, K - done)
        for j in range(chunk):
            ctx.flush_l2()
            ctx.record(2 * j)
            sat.energy_device(ctx, configs, n, d_x, d_s, d_e, d_g, None, threads=threads)
            ctx.record(2 * j + 1)
        for j in range(chunk):
            kernel_ms.append(ctx.elapsed(2 * j, 2 * j + 1))
        done += chunk
    ctx.sync()
    launches = ctx.launches() - launches0
    clk = clocks.stop()
    D.barrier()
    total_ms = D.max(sum(kernel_ms))
    cand_pairs = D.sum(pairs_per_step * K)
    value = cand_pairs / (total_ms / 1e3)
    # the same time counted as all-pairs tests (n (n - 1) / 2 per configuration)
    all_pairs_per_s = D.sum(configs * n * (n - 1) // 2 * K) / (total_ms / 1e3)
    ms_per_step = total_ms / K
    mean_ms = sum(kernel_ms) / len(kernel_ms)

    # end to end through the public host-pointer call: pinned inputs in,
    # energies + gradient back, every step
    hin = N.PinnedArray(x32.shape, np.float32)
    hin.array[...] = x32
    hs = N.PinnedArray((configs,), np.float32)
    hs.array[...] = s32
    he = N.PinnedArray((configs,), np.float32)
    hg = N.PinnedArray(x32.shape, np.float32)
    L = N.lib()
    e2e_steps = max(3, min(K, 200))
    for _ in range(3):
        N.check(L.sqs_sat_energy_host(ctx.handle, configs, n, N.ptr(hin.array, N._fp), N.ptr(hs.array, N._fp),
                                      N.ptr(he.array, N._fp), N.ptr(hg.array, N._fp), None))
    D.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        N.check(L.sqs_sat_energy_host(ctx.handle, configs, n, N.ptr(hin.array, N._fp), N.ptr(hs.array, N._fp),
                                      N.ptr(he.array, N._fp), N.ptr(hg.array, N._fp), None))
    e2e_s = D.max(time.perf_counter() - t0)
    e2e_val = D.sum(pairs_per_step * e2e_steps) / e2e_s
    h2d = x32.nbytes + s32.nbytes
    d2h = configs * 4 + x32.nbytes

    peak, peak_kind = peaks()
    kernel_name = "sat_energy_warp_kernel" if (threads <= 0 and n <= 256) else "sat_energy_kernel"
    algo = algorithmic_bytes(configs, n)
    achieved = algo / (mean_ms / 1e3) / 1e9
    # FP32 work: 55 flop per candidate pair (energy + gradient), against the
    # nominal FP32 peak at the sampled SM clock (148 SMs x 128 lanes x 2)
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
    fp32_achieved = pairs_per_step * 55 / (mean_ms / 1e3) / 1e12
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=D.world, steps=K, warmup=args.warmup,
        ms_per_step=ms_per_step, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
        data="synthetic",
        config=dict(workload=f"SAT energy+gradient, {configs} configs x n={n}, FP32 cell list",
                    configs=configs, n=n, seed=SEED, side=float(s32[0]), l2="flushed before every launch",
                    cta_threads=threads if threads > 0 else 32 * (-threads or 2),
                    kernel_shape=(f"one warp per configuration, {-threads or 2} per CTA" if threads <= 0 and n <= 256
                                  else "one CTA per configuration"),
                    parallelism=f"replicas x{D.world}", device=name, sm_count=sms),
        e2e=dict(value=e2e_val, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                 steps=e2e_steps, call="sqs_sat_energy_host (pinned host buffers)"),
        roofline=dict(bound="issue", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                      traffic=ncu_traffic(kernel_name), peak_kind=peak_kind,
                      algorithmic_bytes_per_launch=algo, kernel=kernel_name,
                      limiter="issue slots: the kernel issues instructions most cycles while DRAM and the FP32 "
                              "pipe are far from their peaks (ncu summary in profiles/)",
                      issue_active_frac=ncu_metric(kernel_name, "issue_active_frac"),
                      hbm=dict(achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak),
                      fp32=dict(achieved=fp32_achieved, peak=fp32_peak, unit="TFLOP/s",
                                frac=fp32_achieved / fp32_peak, peak_kind="nominal at the sampled SM clock",
                                flop_per_candidate_pair=55)),
        gpu_launches=launches,
        pairs_per_step=pairs_per_step,
        all_pairs_equivalent_per_s=all_pairs_per_s,
        clocks=clk,
    )
    if D.rank == 0:
        line["accuracy"] = accuracy(d_e, d_g, x32, s32)
        if not args.no_extras:
            line["anneal_accuracy"] = anneal_accuracy(ctx)
    if D.rank == 0 and D.world == 1 and not args.no_cpu_baseline:
        val, kind, cores, sample, _, _ = cpu_pairs_per_s(x32, s32, args.cpu_seconds)
        line["cpu_baseline"] = dict(value=val, unit=UNIT, cores=cores, kind=kind, sample=sample)
    if D.rank == 0 and D.world == 1 and not args.no_extras:
        line["certify"] = bench_certify(ctx, args.cpu_seconds)
        line["served"] = bench_served_sweep(ctx, args.served_rates, args.served_jobs, args.served_sweeps,
                                            args.served_slice)
        # 10,000 sweeps on a 24-job stream of the full n range, and the
        # configured 50,000 sweeps on an 8-job stream of n <= 100 (a job of
        # n = 1000 alone needs over a minute at 50,000 sweeps)
        line["served_10k"] = bench_served_budget(ctx, 24, 10000)
        line["served_50k"] = bench_served_budget(ctx, 8, 50000, n_hi=100)
        line["plain_pt"] = bench_plain_pt(ctx)
        line["batched"] = bench_batched(ctx)
        # the seeded drop-in against the reference's own seeded program on this GPU
        line["search"] = bench_search()
    for d in (d_x, d_s, d_e, d_g, d_c):
        d.free()
    for h in (hin, hs, he, hg):
        h.free()
    ctx.close()
    if D.rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ extras
def bench_certify(ctx, cpu_seconds: float = 0.0, count: int = 10000):
    """The interval-certifier batch: 10,000 packings, n log-uniform in
    [5, 1000], half exact grids, half tilted near-contact lattices, 5% with
    injected 1e-10 overlaps; GPU end to end from host strings vs the
    reference certifier (certifier.cpp) on all host cores."""
    import numpy as np

    from sqs import core
    from sqs.workloads import certify_corpus

    items = certify_corpus(count, seed=42)
    arrs = core.pack_batch(items)
    squares = int(sum(n for n, _ in items))
    core.certify_arrays(*arrs, ctx=ctx)  # warm-up (first-use set-up)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        out = core.certify_arrays(*arrs, ctx=ctx)
        times.append(time.perf_counter() - t0)
    gpu_s = min(times)
    gpu_ok = np.array([out[k].ok for k in range(count)], np.int32)
    res = dict(workload=f"{count} packings, {squares} squares, n log-uniform [5, 1000]",
               packings_per_s=count / gpu_s, squares_per_s=squares / gpu_s, seconds=gpu_s,
               accepted=int(gpu_ok.sum()), call="sqs_certify_batch (host strings in, verdicts out)")
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    which = "ref" if O.ref_available() else "oracle"
    # the whole batch on the host cores: the CPU baseline and the check of
    # every verdict, reason, score and 50-decimal side
    t0 = time.perf_counter()
    ok, score, Ls, reasons = O.certify_batch_text(*arrs, which=which)
    cpu_s = time.perf_counter() - t0
    used = os.cpu_count() or 1
    same = sum(1 for p in range(count)
               if (int(out[p].ok), float(out[p].score), out[p].L.decode(), out[p].reason.decode()) ==
               (int(ok[p]), float(score[p]), Ls[p], reasons[p]))
    res["cpu_baseline"] = dict(packings_per_s=count / cpu_s, seconds=cpu_s, cores=used,
                               kind="reference" if which == "ref" else "port",
                               sample=f"all {count} packings")
    res["equal_to_reference"] = dict(packings=count, identical=same,
                                     fields="verdict, reason, score, 50-decimal side")
    res["speedup_vs_cpu"] = res["packings_per_s"] / res["cpu_baseline"]["packings_per_s"]
    return res


def served_jobs(count: int, sweeps: int = 2000, n_hi: int = 1000):
    """Anneal-and-certify jobs of the served stream: n log-uniform in
    [5, n_hi], 16, 32 or 64 replicas, a `sweeps` budget each (2,000 by
    default: a bounded stand-in for the configured 50,000 sweeps, whose stream
    of n up to 1000 would not end in a bench run -- one n = 1000 job alone
    takes over a minute at 50,000 sweeps), seeded."""
    import math

    import numpy as np

    from sqs.anneal import AnnealJob, jittered_grid

    rng = np.random.default_rng(7)
    jobs = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(5), math.log(n_hi)))))
        replicas = int(rng.choice([16, 32, 64]))
        xya, L0 = jittered_grid(n, seed=100 + k)
        jobs.append(AnnealJob(xya, L0=L0, replicas=replicas, sweeps=sweeps, exchange_every=10, tmin=1e-3, tmax=1e-1,
                              seed=1000 + k, polish_iters=100))
    return jobs


def bench_served(ctx, jobs, plain, rate: float, slice_proposals: int = 4000, live=None):
    """Served vs plain at one Poisson arrival rate: a stream of about four
    seconds of arrivals (at least 40 jobs, at most all of them) through the
    continuous-batching server; the plain comparator serves the same jobs one
    launch per job in arrival order, its service times measured once
    (`plain`), its latencies from those times and the same arrivals.  The
    same final L is checked job by job."""
    import math

    from sqs.serve import Server, plain_stats, poisson_arrivals, run_stream

    count = min(len(jobs), max(40, int(math.ceil(4 * rate))))
    sub = jobs[:count]
    arr = poisson_arrivals(count, rate, seed=3)
    with Server(ctx, hbm_bytes=4 << 30, max_active=count, slice_proposals=slice_proposals) as srv:
        served, s_stats = run_stream(srv, sub, arr, timeout=600)
        counters = srv.stats()
    p_res, p_service = plain
    p_stats = plain_stats(p_res[:count], p_service[:count], arr)
    if live is not None:
        p_stats["live"] = live
    same_L = all((a or {}).get("L") == (b or {}).get("L") for a, b in zip(served, p_res[:count]))
    # annealing work done per second of the stream: against the batched
    # launch's rate it says how busy the stream kept the GPU
    props = sum(int((r or {}).get("proposals", 0)) for r in served)
    s_stats["proposals_per_s"] = props / s_stats["seconds"] if s_stats["seconds"] > 0 else 0.0
    p_stats["proposals_per_s"] = props / p_stats["seconds"] if p_stats["seconds"] > 0 else 0.0
    return dict(workload=f"{count} jobs, Poisson {rate:g}/s, n log-uniform [5, 1000], 16/32/64 replicas, "
                         f"{jobs[0].sweeps} sweeps", served=s_stats, plain=p_stats, equal_final_L=same_L,
                server_counters=counters,
                served_over_plain=s_stats["certified_jobs_per_s"] / max(p_stats["certified_jobs_per_s"], 1e-12))


def bench_plain_pt(ctx):
    """The plain single-instance PT-SA job: n=10, L0=4, grid + U(+-0.05)
    jitter and U[0, 0.1) angles from seed 42, 8 replicas on 1e-3..1e-1,
    20,000 sweeps, shrink 0.1% per improvement, FP64 polish, certification."""
    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid

    xya, _ = jittered_grid(10, seed=42)
    job = AnnealJob(xya, L0=4.0, replicas=8, sweeps=20000, exchange_every=10, tmin=1e-3, tmax=1e-1, seed=42)
    t0 = time.perf_counter()
    r = anneal_batch([job], ctx=ctx)[0]
    dt = time.perf_counter() - t0
    res = dict(workload="n=10, 8 replicas, 20,000 sweeps", seconds=dt, certified=r["certified"], L=r["L"],
               proposals=r["proposals"], proposals_per_s=r["proposals"] / dt, shrinks=r["shrinks"])
    # the same job on one host core: the CPU annealer of the oracle (O(n)
    # FP64 energy change per proposal, as the reference's search computes it)
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    t0 = time.perf_counter()
    (c,), used = O.ptsa_batch([job], threads=1)
    cs = time.perf_counter() - t0
    res["cpu_baseline"] = dict(proposals_per_s=c["proposals"] / cs, seconds=cs, cores=used, kind="port",
                               best_certified_side=c["best_L"], sample="the whole job (20,000 sweeps)")
    return res


def bench_served_sweep(ctx, rates: str, count: int = 240, sweeps: int = 2000, slice_proposals: int = 4000,
                       live_rate: float = 200.0):
    """Served vs plain at each rate.  The plain comparator is run live once,
    at `live_rate` (its jobs served one launch per job as they arrive); its
    measured per-job service times give the FIFO latencies at the other rates
    (the plain queue never empties, so live and computed agree: both are
    reported at the live rate)."""
    import math

    from sqs.serve import poisson_arrivals, run_plain_live

    rs = [float(x) for x in rates.split(",") if x]
    jobs = served_jobs(count, sweeps)
    need = min(count, max(40, max(int(math.ceil(4 * r)) for r in rs)))
    live_count = min(len(jobs), max(40, int(math.ceil(4 * live_rate))))
    assert live_count >= need or live_count == len(jobs)
    p_res, p_service, p_live = run_plain_live(ctx, jobs[:live_count], poisson_arrivals(live_count, live_rate, seed=3))
    plain = (p_res, p_service)
    out = {f"{r:g}/s": bench_served(ctx, jobs, plain, r, slice_proposals, live=p_live if r == live_rate else None)
           for r in rs}
    out["budget_sweeps"] = sweeps
    return out


def bench_served_budget(ctx, count: int, sweeps: int, n_hi: int = 1000, rate: float = 200.0,
                        slice_proposals: int = 4000):
    """A short stream at a large budget: `count` jobs, n log-uniform in
    [5, n_hi], 16/32/64 replicas, `sweeps` each, Poisson arrivals; served
    against the plain comparator run live."""
    from sqs.serve import Server, poisson_arrivals, run_plain_live, run_stream

    jobs = served_jobs(count, sweeps=sweeps, n_hi=n_hi)
    arr = poisson_arrivals(count, rate, seed=3)
    with Server(ctx, hbm_bytes=4 << 30, max_active=count, slice_proposals=slice_proposals) as srv:
        served, s_stats = run_stream(srv, jobs, arr, timeout=900)
    p_res, _, p_stats = run_plain_live(ctx, jobs, arr)
    same_L = all((a or {}).get("L") == (b or {}).get("L") for a, b in zip(served, p_res))
    return dict(workload=f"{count} jobs, Poisson {rate:g}/s, n log-uniform [5, {n_hi}], 16/32/64 replicas, "
                         f"{sweeps} sweeps", served=s_stats, plain_live=p_stats, equal_final_L=same_L,
                served_over_plain=s_stats["certified_jobs_per_s"] / max(p_stats["certified_jobs_per_s"], 1e-12))


# Algorithmic FP32 work of one proposal, the cost unit 2 k * 35 + 2 * 10 flop
# (the pair energy before and after the move against each of the k squares
# within d^2 < 2 of the moved one, and the two wall terms), with k ~ 4 at
# packing densities: 300 flop.
PROPOSAL_FLOP = 2 * 4 * 35 + 2 * 10


def bench_batched(ctx, sweeps: int = 50, instances: int = 512):
    """Batched PT-SA: 512 instances, n uniform in [20, 400] (seeded), 32
    replicas on 1e-4..5e-2, sigma 0.02 / 0.05 rad, exchange every 10 sweeps,
    FP64 recompute of each best; a bounded sweep budget.  Launch shapes and
    cell sides from the autotuner (tuned once per job class before timing);
    the default fixed shape and the slice loop replayed as a CUDA graph
    (slices of one exchange interval) are timed beside the single launch."""
    from collections import Counter
    from dataclasses import replace

    import numpy as np

    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid

    rng = np.random.default_rng(42)
    jobs = []
    for k in range(instances):
        n = int(rng.integers(20, 401))
        xya, L0 = jittered_grid(n, seed=k)
        jobs.append(AnnealJob(xya, L0=L0, replicas=32, sweeps=sweeps, exchange_every=10, tmin=1e-4, tmax=5e-2,
                              sigma_xy=0.02, sigma_a=0.05, seed=k, polish_iters=0, autotune=True))
    t0 = time.perf_counter()
    anneal_batch([replace(j, sweeps=10) for j in jobs], ctx=ctx)  # tunes every job class, warms up
    tune_s = time.perf_counter() - t0

    def timed(js, slice_sweeps=0):
        g0 = ctx.graph_replays()
        t = time.perf_counter()
        res = anneal_batch(js, ctx=ctx, slice_sweeps=slice_sweeps)
        return res, time.perf_counter() - t, ctx.graph_replays() - g0

    res, dt, _ = timed(jobs)
    fixed, _, _ = timed([replace(j, autotune=False) for j in jobs])
    graph, _, replays = timed(jobs, slice_sweeps=10)
    props = sum(r["proposals"] for r in res)
    dev_s = res[0]["device_ms"] / 1e3
    fixed_s = fixed[0]["device_ms"] / 1e3
    graph_s = graph[0]["device_ms"] / 1e3
    same = all(a[k] == b[k] == c[k] for a, b, c in zip(res, fixed, graph) for k in ("L_cert", "proposals", "accepted"))
    shapes = Counter(f"{r['launch']['cluster_ctas']}x{r['launch']['replicas_per_cta']}/"
                     f"{r['launch']['cell_side']:.2f}" for r in res)
    # CPU baseline: the oracle's annealer on all host threads, a bounded
    # sample of the same jobs (the first 48 instances, 10 sweeps each)
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    sample = [replace(j, sweeps=10) for j in jobs[:48]]
    t0 = time.perf_counter()
    cres, used = O.ptsa_batch(sample, threads=os.cpu_count() or 1)
    cs = time.perf_counter() - t0
    cpu = dict(proposals_per_s=sum(c["proposals"] for c in cres) / cs, seconds=cs, cores=used, kind="port",
               sample="first 48 of the instances, 10 sweeps each")
    return dict(workload=f"{instances} instances, n U[20,400], 32 replicas, {sweeps} sweeps",
                cpu_baseline=cpu, speedup_vs_cpu=(props / dev_s) / cpu["proposals_per_s"],
                proposals=props, seconds=dt, device_seconds=dev_s, proposals_per_s=props / dev_s,
                replica_sweeps_per_s=sum(j.replicas * j.sweeps for j in jobs) / dev_s,
                flops_per_s=props * PROPOSAL_FLOP / dev_s,
                fixed_shape=dict(device_seconds=fixed_s, proposals_per_s=props / fixed_s),
                graph_slices=dict(slice_sweeps=10, graph_replays=replays, device_seconds=graph_s,
                                  proposals_per_s=props / graph_s),
                same_results_all_three=same, tuned_shapes=dict(shapes.most_common()), tune_seconds=tune_s,
                overflows=sum(r["launch"]["overflows"] for r in res),
                squares=int(sum(j.n for j in jobs)) * 32, certified=sum(r["certified"] for r in res))


def bench_search(cases: str = "10:200:64:64,50:60:64:64,200:10:48:64,50:600:64:64,200:100:48:64",
                 prog: str = "seeded"):
    """The search programs head to head on the same B200: this library's
    `seeded` (or `packing`) drop-in and the reference's own program of that
    name (built for sm_100a from its sources into oracle/_ref), same seed file
    (grid centres + U(+-0.05) jitter, angles U[0, 0.1), seed 42, side
    ceil(sqrt n)), epochs, steps, chains and environment (*_AUTOTUNE=0 so both
    keep the chain count).  Reports each program's own seconds, wall time,
    proposals and the side the official gate certifies for its raw result
    (demo.certified_candidate)."""
    import subprocess
    import tempfile

    from sqs.anneal import jittered_grid
    from sqs.demo import certified_candidate

    if prog not in ("seeded", "packing"):
        raise ValueError(f"unknown search program {prog!r}")
    progs = {"sqs": ROOT / "squares-in-squares_b200" / "bin" / prog,
             "reference": ROOT / "oracle" / "_ref" / prog}
    env = dict(os.environ, **{"SEED_AUTOTUNE" if prog == "seeded" else "PACK_AUTOTUNE": "0"})
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for case in cases.split(","):
            n, epochs, steps, chains = (int(v) for v in case.split(":"))
            xya, L = jittered_grid(n, seed=42)
            seed = Path(tmp) / f"seed{n}.txt"
            seed.write_text(f"{n} {L}\n" + "".join(f"{x:.17g} {y:.17g} {a:.17g}\n" for x, y, a in xya))
            row = {}
            for name, exe in progs.items():
                if not exe.exists():
                    row[name] = dict(unavailable=f"{exe.name} not built")
                    continue
                res = Path(tmp) / f"{name}{n}.json"
                # a one-step warm-up run first, so neither program's wall time
                # holds the first load of its binary and libraries
                subprocess.run([str(exe), str(seed), "1", "1", "8", "7", str(res)], capture_output=True, env=env,
                               timeout=300)
                t0 = time.perf_counter()
                r = subprocess.run([str(exe), str(seed), str(epochs), str(steps), str(chains), "7", str(res)],
                                   capture_output=True, text=True, env=env, timeout=600)
                wall = time.perf_counter() - t0
                if r.returncode != 0:
                    row[name] = dict(exit=r.returncode, stderr=r.stderr[-300:])
                    continue
                raw = json.loads(res.read_text())
                try:
                    _, side, dil = certified_candidate(raw)
                except ValueError as e:
                    side, dil = None, str(e)
                row[name] = dict(seconds=raw["seconds"], wall_seconds=wall, proposals=raw["proposals"],
                                 proposals_per_s=raw["proposals"] / max(raw["seconds"], 1e-9),
                                 target_L=raw["target_L"], certified_L=side, dilation=dil, chains=raw["chains"])
            if "seconds" in row.get("sqs", {}) and "seconds" in row.get("reference", {}):
                row["wall_speedup"] = row["reference"]["wall_seconds"] / row["sqs"]["wall_seconds"]
            out[f"{prog} n={n} epochs={epochs} steps={steps} chains={chains}"] = row
    return out


def bench_batched_fixed(ctx, sweeps: int, instances: int):
    """The batched workload at the default launch shapes (no autotuner, one
    call): a clean single launch per cluster shape, for profiling."""
    import numpy as np

    from sqs.anneal import AnnealJob, anneal_batch, jittered_grid

    rng = np.random.default_rng(42)
    jobs = []
    for k in range(instances):
        n = int(rng.integers(20, 401))
        xya, L0 = jittered_grid(n, seed=k)
        jobs.append(AnnealJob(xya, L0=L0, replicas=32, sweeps=sweeps, exchange_every=10, tmin=1e-4, tmax=5e-2,
                              sigma_xy=0.02, sigma_a=0.05, seed=k, polish_iters=0))
    res = anneal_batch(jobs, ctx=ctx)
    props = sum(r["proposals"] for r in res)
    dev_s = res[0]["device_ms"] / 1e3
    return dict(workload=f"{instances} instances, n U[20,400], 32 replicas, {sweeps} sweeps, default shapes",
                proposals=props, device_seconds=dev_s, proposals_per_s=props / dev_s)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("sqs", "reference"), default="sqs")
    ap.add_argument("--threads", type=int, default=0, help="CTA width (0 = library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the certifier / served / plain-PT / batched sections")
    ap.add_argument("--section", choices=("certify", "served", "served_full", "plain_pt", "batched", "batched_fixed",
                                          "search", "anneal_accuracy"),
                    help="run only this extra section (for profiling) and print its dict")
    ap.add_argument("--batched-instances", type=int, default=512)
    ap.add_argument("--batched-sweeps", type=int, default=50)
    ap.add_argument("--served-rates", default="200,1000")
    ap.add_argument("--served-jobs", type=int, default=240, help="most jobs in one served stream")
    ap.add_argument("--served-sweeps", type=int, default=2000, help="sweep budget of every served job")
    ap.add_argument("--served-slice", type=int, default=4000, help="proposals per replica per server slice")
    ap.add_argument("--search-prog", choices=("seeded", "packing"), default="seeded",
                    help="which search program the search section compares")
    args = ap.parse_args()
    if args.section:
        from sqs import Context

        with Context(int(os.environ.get("LOCAL_RANK", 0))) as ctx:
            fn = dict(certify=lambda: bench_certify(ctx, args.cpu_seconds),
                      served=lambda: bench_served_sweep(ctx, args.served_rates, args.served_jobs,
                                                        args.served_sweeps, args.served_slice),
                      served_full=lambda: dict(served_10k=bench_served_budget(ctx, 24, 10000),
                                               served_50k=bench_served_budget(ctx, 8, 50000, n_hi=100),
                                               served_50k_full_range=bench_served_budget(ctx, 16, 50000)),
                      plain_pt=lambda: bench_plain_pt(ctx),
                      batched=lambda: bench_batched(ctx, args.batched_sweeps, args.batched_instances),
                      batched_fixed=lambda: bench_batched_fixed(ctx, args.batched_sweeps, args.batched_instances),
                      search=lambda: bench_search(prog=args.search_prog),
                      anneal_accuracy=lambda: anneal_accuracy(ctx))[args.section]
            print(json.dumps({args.section: fn()}), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3
    D = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, D)
        else:
            run_sqs(args, D)
    finally:
        D.close()


if __name__ == "__main__":
    main()
