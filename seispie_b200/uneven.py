"""Uneven-size batches: many independent models stepped together.

Each instance has its own grid, model, sources (one per shot), receivers
and nt.  Instances of one wave type share one launch per time step
(fwi_multi_run); the whole time loop of every wave type can be captured into
one CUDA graph and replayed as a single launch.

    python -m seispie_b200.uneven [--instances 48] [--seed 0]

runs the uneven-batch configuration (48 SH and P-SV instances, grids drawn
from 128 to 768 cells a side with aspect 1:1 to 2:1, nt 1500-6000, 8-32
shots, smooth-plus-checkerboard models seeded per instance) and prints one
JSON line: throughput and HBM roofline of the step launches.  The traces'
errors against the FP64 oracle are checked by tests/test_gpu_uneven.py.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, engine
from ._lib import FwiBatch, check
from .engine import Grid, ShotBatch, build_model, injection_lists, point_ids, ricker_stf


@dataclass
class Instance:
    mode: str
    nx: int
    nz: int
    h: float
    dt: float
    nt: int
    params: dict          # rho, vp, vs (host float32, reference cell order)
    src: np.ndarray       # [nshots, 7] source lines (one shot per source)
    rec: np.ndarray       # [nrec, 2]
    absorb: tuple = (20, 0.015, 1, 1, 1, 0)
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.nz * self.nt * len(self.src)


def make_instances(n: int = 48, seed: int = 0, sizes=(128, 768), nts=(1500, 6000), shots=(8, 32),
                   nrec_per_cell: float = 0.25) -> list[Instance]:
    """Seeded synthetic instances of the uneven-batch configuration."""
    out = []
    for k in range(n):
        rng = np.random.default_rng(seed * 100003 + k)
        mode = "sh" if k % 2 == 0 else "psv"
        nz = int(rng.integers(sizes[0], sizes[1] + 1))
        nx = int(min(sizes[1], round(nz * rng.uniform(1.0, 2.0))))
        nt = int(rng.integers(nts[0], nts[1] + 1))
        ns = int(rng.integers(shots[0], shots[1] + 1))
        i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        sq = int(rng.integers(16, 65))
        board = np.where(((i // sq) + (j // sq)) % 2 == 0, 1.0, -1.0)
        smooth = np.sin(rng.uniform(1, 3) * i / nx + rng.uniform(0, 6)) * np.cos(rng.uniform(1, 3) * j / nz)
        vp = (3000 * (1 + 0.04 * smooth + 0.05 * board)).astype(np.float32).ravel()
        vs = (vp / np.sqrt(3.0)).astype(np.float32)
        rho = (2600 * (1 + 0.03 * smooth)).astype(np.float32).ravel()
        h = 10.0
        f0 = 10.0
        src = np.array([[(s + 0.5) * nx / ns * h, 10 * h, 0, f0, 1.2 / f0, 0.0 if mode == "sh" else 15.0, 1e10]
                        for s in range(ns)])
        nrec = max(8, int(nx * nrec_per_cell))
        rec = np.array([[(r + 0.5) * nx / nrec * h, 12 * h] for r in range(nrec)])
        out.append(Instance(mode, nx, nz, h, 1e-3, nt, dict(vp=vp, vs=vs, rho=rho), src, rec, seed=k))
    return out


class UnevenBatch:
    """Device state of a set of instances, grouped by wave type."""

    def __init__(self, instances: list[Instance], tile: int = 0, device="cuda"):
        self.instances = instances
        self.tile = tile
        self.lib = _lib.load()
        self.items = []
        for inst in instances:
            g = Grid(inst.nx, inst.nz, float(np.float32(inst.h)), float(np.float32(inst.h)))
            m = build_model(inst.mode, g, inst.dt, inst.params, inst.absorb, device)
            sid = point_ids(inst.src, np.float32(inst.h), np.float32(inst.h), inst.nz)
            rid = point_ids(inst.rec, np.float32(inst.h), np.float32(inst.h), inst.nz)
            b = ShotBatch(m, len(sid), inst.nt, rid, tile=tile, displacement=True)
            stf, par = ricker_stf(inst.src, inst.nt, inst.dt, device)
            d = b.desc(inj=injection_lists(len(sid), sid, lambda s: s), stf=stf)
            d._stf = (stf, par)
            self.items.append((inst, m, b, d))
        self.groups = {}
        for mode in ("sh", "psv"):
            sel = [it for it in self.items if it[0].mode == mode]
            if not sel:
                continue
            arr = (ctypes.POINTER(FwiBatch) * len(sel))(*[ctypes.pointer(it[3]) for it in sel])
            nbytes = int(self.lib.fwi_multi_workspace_bytes(len(sel)))
            ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
            self.groups[mode] = (sel, arr, ws)
        self.graph = None

    def prepare(self):
        for sel, arr, ws in self.groups.values():
            check(self.lib.fwi_multi_prepare(arr, len(sel), ws.data_ptr()), "fwi_multi_prepare")

    def clear(self):
        for inst, m, b, d in self.items:
            b.clear()
            d.cur = 0

    def run(self):
        s = engine.stream_handle(None)
        for sel, arr, ws in self.groups.values():
            ntmax = max(it[0].nt for it in sel)
            check(self.lib.fwi_multi_run(arr, len(sel), ws.data_ptr(), 0, ntmax, s), "fwi_multi_run")
        for inst, m, b, d in self.items:
            b.cur = d.cur

    def check(self) -> None:
        """Wait for the work queued so far and raise FwiError if a bounded
        wait in a step kernel gave up (engine.check_device)."""
        engine.check_device(None, "UnevenBatch")

    def capture(self):
        """Record clear + every step of every group into one CUDA graph."""
        self.clear()
        self.prepare()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self.clear()
                self.run()
        torch.cuda.current_stream().wait_stream(side)
        self.graph = g
        return g

    def launch_count_per_run(self) -> int:
        return sum(max(it[0].nt for it in sel) for sel, _, _ in self.groups.values())

    def traces(self, k: int):
        """Traces of instance k per component slot, [nshots, nrec, nt]."""
        inst, m, b, d = self.items[k]
        return [b.traces(c) if b.obs[c] is not None else None for c in range(3)]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=48)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--reps", type=int, default=1)
    a = ap.parse_args(argv)
    insts = make_instances(a.instances, a.seed)
    ub = UnevenBatch(insts, tile=a.tile)
    g = ub.capture()
    g.replay()  # warm-up
    torch.cuda.synchronize()
    n0 = ub.lib.fwi_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / a.reps
    cells = sum(i.cells for i in insts)
    bytes_ = sum(i.cells * (44 if i.mode == "sh" else 72) for i in insts)
    peak = 6650.0
    try:
        peak = float(json.load(open(os.path.join(os.path.dirname(os.path.dirname(__file__)),
                                                 "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        pass
    line = {"metric": "Gcell-updates/s (uneven batch, one graph launch)", "value": cells / sec / 1e9,
            "unit": "Gcell-updates/s", "instances": len(insts), "cells": cells, "seconds": sec,
            "graph_launches_per_run": 1, "kernel_launches_per_run": ub.launch_count_per_run(),
            "roofline": {"bound": "hbm", "achieved": bytes_ / sec / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_ / sec / 1e9 / peak},
            "per_instance": [dict(mode=i.mode, nx=i.nx, nz=i.nz, nt=i.nt, shots=len(i.src)) for i in insts]}
    print(json.dumps(line))
    return line


if __name__ == "__main__":
    main()
