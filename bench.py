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
        self.path = ROOT / "gpurun_out" / f".clocks_{os.getpid()}.csv"

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
    all_pairs = D.sum(pairs_per_step * K)
    value = all_pairs / (total_ms / 1e3)
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
    algo = algorithmic_bytes(configs, n)
    achieved = algo / (mean_ms / 1e3) / 1e9
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=D.world, steps=K, warmup=args.warmup,
        ms_per_step=ms_per_step, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
        data="synthetic",
        config=dict(workload=f"SAT energy+gradient, {configs} configs x n={n}, FP32 cell list",
                    configs=configs, n=n, seed=SEED, side=float(s32[0]), l2="flushed before every launch",
                    cta_threads=threads or 64, parallelism=f"replicas x{D.world}", device=name, sm_count=sms),
        e2e=dict(value=e2e_val, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                 steps=e2e_steps, call="sqs_sat_energy_host (pinned host buffers)"),
        roofline=dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                      traffic=ncu_traffic("sat_energy_kernel"), peak_kind=peak_kind,
                      algorithmic_bytes_per_launch=algo, kernel="sat_energy_kernel"),
        gpu_launches=launches,
        pairs_per_step=pairs_per_step,
        clocks=clk,
    )
    if D.rank == 0 and D.world == 1 and not args.no_cpu_baseline:
        val, kind, cores, sample, _, _ = cpu_pairs_per_s(x32, s32, args.cpu_seconds)
        line["cpu_baseline"] = dict(value=val, unit=UNIT, cores=cores, kind=kind, sample=sample)
    for d in (d_x, d_s, d_e, d_g, d_c):
        d.free()
    for h in (hin, hs, he, hg):
        h.free()
    ctx.close()
    if D.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("sqs", "reference"), default="sqs")
    ap.add_argument("--threads", type=int, default=0, help="CTA width (0 = library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    args = ap.parse_args()
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
