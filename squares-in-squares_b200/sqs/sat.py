"""FP32 cell-list SAT overlap energy and gradient on the GPU.

The batched form of the reference's energy model -- walls plus the sum over
pairs of the squared separating-axis penetration (seeded.cu:41-65, 96-113,
148-162) -- for many independent configurations in one launch.
"""
from __future__ import annotations

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
