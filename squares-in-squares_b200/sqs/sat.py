"""FP32 cell-list SAT overlap energy and gradient on the GPU.

The batched form of the reference's energy model -- walls plus the sum over
pairs of the squared separating-axis penetration (seeded.cu:41-65, 96-113,
148-162) -- for many independent configurations in one launch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def energy(xya, side, *, ctx: N.Context | None = None, grad: bool = True, count: bool = False):
    """Energy (and gradient, candidate-pair counts) of a batch, host arrays.

    xya: (configs, n, 3) float32-convertible (x, y, angle); side: scalar or
    (configs,).  Returns (energy[configs], grad[configs, n, 3] | None,
    cand[configs] | None) where cand counts pairs with centre distance^2 < 2.
    """
    xya = np.ascontiguousarray(xya, dtype=np.float32)
    if xya.ndim == 2:
        xya = xya[None]
    configs, n, three = xya.shape
    if three != 3:
        raise ValueError("xya must have shape (configs, n, 3)")
    side = np.ascontiguousarray(np.broadcast_to(np.asarray(side, dtype=np.float32), (configs,)))
    e = np.zeros(configs, np.float32)
    g = np.zeros_like(xya) if grad else None
    c = np.zeros(configs, np.uint32) if count else None
    own = ctx is None
    ctx = ctx or N.Context(0)
    try:
        N.check(N.lib().sqs_sat_energy_host(ctx.handle, configs, n, N.ptr(xya, N._fp), N.ptr(side, N._fp),
                                            N.ptr(e, N._fp), N.ptr(g, N._fp), N.ptr(c, N._u32p)))
    finally:
        if own:
            ctx.close()
    return e, g, c


def energy_device(ctx: N.Context, configs: int, n: int, xya: N.DeviceArray, side: N.DeviceArray,
                  out: N.DeviceArray, grad: N.DeviceArray | None = None,
                  cand: N.DeviceArray | None = None, threads: int = 0) -> None:
    """Launch on device-resident buffers (stream-ordered, no synchronisation)."""
    N.check(N.lib().sqs_sat_energy(ctx.handle, configs, n, xya.ptr, side.ptr, out.ptr,
                                   grad.ptr if grad is not None else None,
                                   cand.ptr if cand is not None else None, threads))


def energy_fp64(states, sides, *, ctx: N.Context | None = None, grad: bool = True):
    """FP64 energy (and gradient) of packings of any sizes (sqs_energy_fp64):
    walls plus pairs, all pairs, with the polish's smooth gradient.

    states: list of (n_k, 3) arrays (or one (configs, n, 3) array); sides:
    scalar or one per packing.  Returns (energy float64[count], list of
    (n_k, 3) gradients | None)."""
    if isinstance(states, np.ndarray) and states.ndim == 3:
        states = list(states)
    states = [np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 3) for q in states]
    count = len(states)
    n_of = np.array([q.shape[0] for q in states], dtype=np.int32)
    flat = np.ascontiguousarray(np.concatenate(states, axis=0)) if count else np.zeros((0, 3))
    side = np.ascontiguousarray(np.broadcast_to(np.asarray(sides, dtype=np.float64), (count,)))
    e = np.zeros(count)
    g = np.zeros_like(flat) if grad else None
    own = ctx is None
    ctx = ctx or N.Context(0)
    try:
        N.check(N.lib().sqs_energy_fp64(ctx.handle, count, N.ptr(n_of, C.POINTER(C.c_int32)),
                                        N.ptr(flat, N._dp), N.ptr(side, N._dp), N.ptr(e, N._dp),
                                        N.ptr(g, N._dp)))
    finally:
        if own:
            ctx.close()
    if g is None:
        return e, None
    return e, np.split(g, np.cumsum(n_of)[:-1])
