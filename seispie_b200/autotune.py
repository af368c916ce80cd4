"""Tile-shape autotuner for the fused step kernel.

Times every step-kernel variant the library offers (``fwi_tile_shape``) on
the caller's own batch shape -- forward steps on scratch wavefields, timed
with CUDA events on the current stream -- and returns the fastest.  Results
are cached per (wave type, grid, shots, receivers) for the process.
"""
from __future__ import annotations

import torch

from . import _lib
from .engine import DeviceModel, ShotBatch

_CACHE: dict[tuple, tuple[int, dict[int, float]]] = {}


def autotune(model: DeviceModel, nshots: int, nt: int, rec_id, inj, stf, steps: int = 60, warm: int = 10,
             variants=None) -> tuple[int, dict[int, float]]:
    """Return (best tile variant, {variant: ms per forward step})."""
    g = model.grid
    key = (model.mode, g.nx, g.nz, nshots, len(rec_id))
    if key in _CACHE and variants is None:
        return _CACHE[key]
    steps = max(1, min(steps, nt - warm))
    times: dict[int, float] = {}
    for t in variants or _lib.tile_variants():
        b = ShotBatch(model, nshots, nt, rec_id, tile=t, displacement=True)
        d = b.desc(inj=inj, stf=stf)
        b.clear()
        b.run(d, False, 0, min(warm, nt))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run(d, False, min(warm, nt - steps), steps)
        e1.record()
        torch.cuda.synchronize()
        times[t] = e0.elapsed_time(e1) / steps
        del b, d
    best = min(times, key=times.get)
    if variants is None:
        _CACHE[key] = (best, times)
    return best, times
