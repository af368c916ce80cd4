"""Exact gradients of seismograms with respect to the model, and the
``torch.autograd.Function`` around them.

The forward is the fused step (``fwi_run``); the backward is its exact
discrete transpose (``fwi_run_transposed``), which needs, for every step, the
strain of the forward velocity after the step and the stress divergence of
the step.  Those are recomputed segment by segment from checkpoints of the
full wavefield taken every ``K`` steps during the forward pass (uniform
checkpointing): the memory is ``nt/K`` wavefield copies plus ``K`` steps of
strain and divergence, the cost one extra forward sweep.  ``K`` defaults to the value
that balances the two, shrunk further to fit the memory budget.

The reference's own adjoint (solver.py:290-329) is a subsampled continuous
adjoint; ``seispie_b200.solver.b200.run_kernel`` reproduces that one.  This
module is what makes finite-difference-exact gradients (and therefore
autograd) possible.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import engine
from ._lib import FWI_PSV, FWI_SH, FWI_SPIN
from .engine import COMP, NS, NV, DeviceModel, Grid, ShotBatch, adjoint_injection_lists, injection_lists


def strain_fields(mode: int) -> int:
    """Stress-update terms stored per step for the gradient (SH exy, ezy;
    P-SV exx, ezz, exz+ezx; spin adds -vy_c - (ezx-exz)/2, Dx+ vy_c, Dz+ vy_c)."""
    return 2 if mode == FWI_SH else 3 if mode == FWI_PSV else 6


def state_fields(mode: int, grid: Grid) -> int:
    """Fields of one checkpoint: stress and velocity, plus the displacement
    where the forward keeps it (engine.displacement_free_ok)."""
    return NS[mode] + (1 if engine.displacement_free_ok(mode, grid) else 2) * NV[mode]


def step_fields(mode: int, density: bool = True) -> int:
    """Fields stored per step for the transposed step: the stress-update
    terms, plus the divergences where the density terms are wanted."""
    return strain_fields(mode) + (NV[mode] if density else 0)


def default_segment(nt: int, mode: int, nshots: int, grid: Grid, budget_bytes: float | None = None,
                    density: bool = True, overlap: bool = False) -> int:
    """Segment length K minimising checkpoint + segment memory
    (nt/K * S fields + B * K * P fields: S = state_fields, P = step_fields,
    B = 1 segment buffer, 2 with overlap), then shrunk to the budget."""
    state = state_fields(mode, grid)
    per_step = step_fields(mode, density) * (2 if overlap else 1)
    k = max(1, int(round(math.sqrt(nt * state / per_step))))
    if budget_bytes:
        field = 4 * nshots * grid.nx * grid.pitch
        while k > 1 and (math.ceil(nt / k) * state + k * per_step) * field > budget_bytes:
            k = max(1, k // 2)
    return min(k, nt)


def fixed_bytes(nt: int, mode: int, nshots: int, grid: Grid, nrec: int = 0, segment: int | None = None,
                overlap: bool = False, density: bool = True) -> int:
    """Upper bound of the device bytes an ExactAdjoint (levels = 1) holds
    besides its stored tail: checkpoints every K steps over all nt steps, one
    segment of per-step stores (two with overlap), the wavefields of the
    forward and adjoint batches (ping-pong stress and velocity, displacement
    where kept) and, per velocity component, the traces, the observed data
    and the trace gradients.  A stored tail has to fit in what is left."""
    k = segment or default_segment(nt, mode, nshots, grid, density=density, overlap=overlap)
    field = 4 * nshots * grid.nx * grid.pitch
    state = state_fields(mode, grid)
    per_step = step_fields(mode, density)
    batch = 2 * NS[mode] + 2 * NV[mode] + (state - NS[mode] - NV[mode])
    segs = 2 if overlap else 1
    return ((math.ceil(nt / k) * state + segs * k * per_step + 2 * batch) * field
            + 3 * 4 * nshots * nrec * nt * NV[mode])


def max_tail_bytes(nt: int, mode: int, nshots: int, grid: Grid, budget_bytes: float, nrec: int = 0,
                   segment: int | None = None, overlap: bool = False, density: bool = True) -> int:
    """Largest stored tail (as ExactAdjoint's tail_memory, in bytes) whose
    ExactAdjoint (levels = 1) fits budget_bytes in all: checkpoints of the
    steps before the tail, one segment of per-step stores (two with
    overlap), the tail's per-step stores, both batches' wavefields and the
    trace arrays (the terms of fixed_bytes).  A longer tail needs fewer
    checkpoints."""
    k = segment or default_segment(nt, mode, nshots, grid, density=density, overlap=overlap)
    field = 4 * nshots * grid.nx * grid.pitch
    state = state_fields(mode, grid)
    per_step = step_fields(mode, density)
    batch = 2 * NS[mode] + 2 * NV[mode] + (state - NS[mode] - NV[mode])
    traces = 3 * 4 * nshots * nrec * nt * NV[mode]
    segs = 2 if overlap else 1

    def need(t):
        return (math.ceil((nt - t) / k) * state + segs * k * per_step + t * per_step + 2 * batch) * field + traces

    lo, hi = 0, nt  # need() grows with t: the largest t with need(t) <= budget
    if need(0) > budget_bytes:
        return 0
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if need(mid) <= budget_bytes:
            lo = mid
        else:
            hi = mid - 1
    return lo * per_step * field


def two_level_segments(nt: int, mode: int) -> tuple:
    """(K1, K2) minimising the memory of two-level checkpointing,
    nt/K1 + K1/K2 checkpoints of S = NS+2NV fields plus K2 steps of
    P = NE+NV stored fields: K2 = (S/P)^(2/3) nt^(1/3), K1 = sqrt(nt K2)."""
    S = NS[mode] + 2 * NV[mode]
    P = strain_fields(mode) + NV[mode]
    k2 = max(1, int(round((S / P) ** (2.0 / 3.0) * nt ** (1.0 / 3.0))))
    k1 = max(k2, int(round(math.sqrt(nt * k2))))
    return min(k1, nt), min(k2, nt)


class ExactAdjoint:
    """Forward with checkpoints, then exact backward, for one batch of shots.

    levels = 1: a checkpoint every K steps; the backward recomputes each
    segment once with the per-step stores (one extra forward sweep).
    levels = 2: checkpoints every K1 = `segment` steps; the backward
    recomputes a segment once to lay sub-checkpoints every K2 =
    `sub_segment` steps inside it, then each sub-segment with the per-step
    stores (two extra forward sweeps, memory nt/K1 + K1/K2 checkpoints and K2
    steps of stores instead of nt/K checkpoints and K steps) -- recursive
    checkpointing in the manner of revolve, two levels deep.  Both give the
    same gradient bit for bit.

    tail_memory (bytes): HBM the forward sweep may fill with the per-step
    stores of its last steps; those steps are then transposed without being
    recomputed (exactly the same values, so the same gradient), and only the
    steps before them are checkpointed.

    overlap (levels = 1): two segments of per-step stores; the backward
    recomputes segment s-1 on a second stream while the transposes of
    segment s run, so that the two kernels share the SMs (same values, so
    the same gradient bit for bit); overlap_ctas caps the resident CTAs per
    SM of the recomputing row-marching step (0: no cap), leaving room for
    the transposed step's CTAs.

    density = False: no density terms (backward returns None for dL/dbuo,
    and for spin dL/dbuo_j), so no divergence is stored per step: a P-SV
    step stores 3 fields instead of 5, the stored tail holds 5/3 as many
    steps, and the lambda / mu terms are the same bit for bit.

    step_overlap: programmatic dependent launch between consecutive steps
    (fwi_batch.step_overlap) wherever a time loop has the GPU to itself --
    the forward sweep and a serial backward; the overlapped backward's two
    streams launch without it (measured at 512 x 512 x 32 shots: forward
    sweep 93.3 against 95.8 us per step, overlapped backward 176.8 us per
    step without it against 181-184 with it on either stream).  Same values
    bit for bit either way."""

    def __init__(self, model: DeviceModel, nt: int, src_id, isrc_of_shot, nshots: int, stf, rec_id,
                 segment: int | None = None, tile: int = 0, levels: int = 1, sub_segment: int | None = None,
                 tail_memory: float = 0.0, overlap: bool = False, overlap_ctas: int = 0, density: bool = True,
                 step_overlap: bool = True):
        self.model, self.nt, self.nshots = model, int(nt), int(nshots)
        self.step_overlap = int(bool(step_overlap))
        self.rec_id = np.asarray(rec_id, np.int32)
        self.mode = model.mode
        g = model.grid
        if levels not in (1, 2):
            raise ValueError("levels must be 1 or 2")
        if overlap and levels != 1:
            raise ValueError("overlap needs levels = 1")
        self.levels = levels
        if levels == 1:
            self.K = segment or default_segment(self.nt, self.mode, self.nshots, g, density=density, overlap=overlap)
            self.K2 = self.K
        else:
            k1, k2 = two_level_segments(self.nt, self.mode)
            self.K = segment or k1
            self.K2 = min(sub_segment or k2, self.K)
        field = 4 * self.nshots * g.nx * g.pitch
        self.density = bool(density)
        per_step = step_fields(self.mode, self.density) * field
        self.tail = min(self.nt, int(max(0.0, tail_memory) // per_step))
        self.t0 = self.nt - self.tail  # steps [t0, nt) keep their stores from the forward sweep
        self.nseg = math.ceil(self.t0 / self.K)
        self.fwd = ShotBatch(model, self.nshots, self.nt, self.rec_id, tile=tile)
        # a list to collect (start, end, steps) CUDA events of the checkpointed forward segments
        # (plain steps, no stores), or None
        self.step_events = None
        inj = injection_lists(self.nshots, src_id, isrc_of_shot)
        self.fwd.step_overlap = self.step_overlap
        self.fdesc = self.fwd.desc(inj=inj, stf=stf)
        # recomputed steps record no traces (the forward sweep has them)
        self.rdesc = self.fwd.desc(inj=inj, stf=stf, record=False)
        dev = model.device
        shape = (self.nshots, g.nx, g.pitch)
        nstate = len(self.fwd.state_tensors())
        self.ckpt = torch.empty((self.nseg, nstate) + shape, dtype=torch.float32, device=dev)
        self.ckpt2 = (torch.empty((math.ceil(self.K / self.K2), nstate) + shape, dtype=torch.float32, device=dev)
                      if levels == 2 else None)
        self.seg_e = [None] * 6
        self.seg_ds = [None, None, None]
        for k in range(strain_fields(self.mode)):
            self.seg_e[k] = torch.empty((self.K2,) + shape, dtype=torch.float32, device=dev)
        for c in COMP[self.mode][: NV[self.mode]] if self.density else ():
            self.seg_ds[c] = torch.empty((self.K2,) + shape, dtype=torch.float32, device=dev)
        self.overlap = bool(overlap) and self.nseg > 1
        self.overlap_ctas = int(overlap_ctas)
        self.adj_tile = 0  # P-SV transposed step: 0 = 32 x 64 tiles, 1 = 32 x 32 tiles (same values)
        if self.overlap:
            self.seg_e2 = [None if t is None else torch.empty_like(t) for t in self.seg_e]
            self.seg_ds2 = [None if t is None else torch.empty_like(t) for t in self.seg_ds]
        self._adj = None  # adjoint batch and its injection lists (made by the first backward)
        self._side = None  # the overlapped backward's recomputing stream
        self.tail_e, self.tail_ds = [None] * 6, [None, None, None]
        if self.tail:
            for k in range(strain_fields(self.mode)):
                self.tail_e[k] = torch.empty((self.tail,) + shape, dtype=torch.float32, device=dev)
            for c in COMP[self.mode][: NV[self.mode]] if self.density else ():
                self.tail_ds[c] = torch.empty((self.tail,) + shape, dtype=torch.float32, device=dev)

    def forward(self) -> list:
        """Run the forward, keeping a checkpoint every K steps; returns the
        traces per component slot (None where absent), [nshots, nrec, nt].
        Also sums, over every checkpoint and shot, the squared particle
        velocity into self.illum (FP64 [nx, pitch]): the source illumination
        the learned preconditioner reads."""
        b = self.fwd
        b.clear()
        g = self.model.grid
        self.illum = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.model.device)
        for s in range(self.nseg):
            for q, t in enumerate(b.state_tensors()):
                self.ckpt[s, q].copy_(t)
            for v in b.vel[b.cur]:
                engine.energy_accumulate(v, self.illum)
            n = min(self.K, self.t0 - s * self.K)
            if self.step_events is not None:  # CUDA events around the plain forward steps
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(torch.cuda.current_stream() if b.stream is None else b.stream)
            b.run(self.fdesc, False, s * self.K, n)
            if self.step_events is not None:
                e1.record(torch.cuda.current_stream() if b.stream is None else b.stream)
                self.step_events.append((e0, e1, n))
        if self.tail:
            # the illumination is sampled at the multiples of K whatever the tail, so that it does not
            # depend on how much memory the tail got
            b.set_segment(self.fdesc, self.tail_e, self.tail_ds, self.t0, self.tail)
            s0 = self.t0
            while s0 < self.nt:
                if s0 % self.K == 0:
                    for v in b.vel[b.cur]:
                        engine.energy_accumulate(v, self.illum)
                s1 = min(self.nt, (s0 // self.K + 1) * self.K)
                b.run(self.fdesc, False, s0, s1 - s0)
                s0 = s1
            b.set_segment(self.fdesc, [None] * 6, [None] * 3, 0, 0)
        return [b.traces(c).clone() if b.obs[c] is not None else None for c in range(3)]

    def backward(self, g_traces: list) -> tuple:
        """Exact gradients from trace gradients (per component slot, each
        [nshots, nrec, nt] in forward time order).  Returns FP64
        (dL/dlam, dL/dmu, dL/dbuo) on [nx, pitch] (dL/dlam is zero for SH);
        spin adds (dL/dnu, dL/dmnc, dL/dbuo_j) with mnc = mu_c + nu_c and
        buo_j = dt/j.  Spin losses may depend on ux and uz only.  Without
        density terms (density = False) dL/dbuo and dL/dbuo_j are None."""
        if self.mode == FWI_SPIN and g_traces[1] is not None:
            raise ValueError("the spin adjoint injects x and z trace gradients only (no uy_c term)")
        gr = self.model.grid
        dev = self.model.device
        k = [torch.zeros((gr.nx, gr.pitch), dtype=torch.float64, device=dev)
             for _ in range(6 if self.mode == FWI_SPIN else 3)]
        if not self.density:  # the buoyancy slots: dL/dbuo (2) and, for spin, dL/dbuo_j (5)
            for q in ((2, 5) if self.mode == FWI_SPIN else (2,)):
                k[q] = None
        stf = [None, None, None]
        for c in range(3):
            if g_traces[c] is not None and self.fwd.obs[c] is not None:
                # u~ at the receivers: suffix sums of dL/d(trace) over time
                g = g_traces[c].to(torch.float32).contiguous()
                stf[c] = engine.trace_suffix_sum(g, torch.empty_like(g)).reshape(-1)
        adj, inj = self._adjoint_batch()
        adj.adj_tile = self.adj_tile
        # the overlapped backward's streams share the SMs: no early launches there
        adj.step_overlap = 0 if self.overlap else self.step_overlap
        adj.clear()
        adesc = adj.desc(inj=inj, stf=stf, record=False, kernels=k)
        fwd = self.fwd

        def reverse(t0, n):
            """Recompute steps [t0, t0+n) from the current state with the
            per-step stores and run their transposes."""
            fwd.set_segment(self.rdesc, self.seg_e, self.seg_ds, t0, n)
            fwd.run(self.rdesc, False, t0, n)
            adj.set_segment(adesc, self.seg_e, self.seg_ds, t0, n)
            adj.run_transposed(adesc, t0 + n, n)

        if self.overlap:
            self._backward_overlapped(adj, adesc)
            return tuple(k)
        if self.tail:
            adj.set_segment(adesc, self.tail_e, self.tail_ds, self.t0, self.tail)
            adj.run_transposed(adesc, self.nt, self.tail)
        for s in reversed(range(self.nseg)):
            s0, n = s * self.K, min(self.K, self.t0 - s * self.K)
            for q, t in enumerate(fwd.state_tensors()):
                t.copy_(self.ckpt[s, q])
            if self.levels == 1:
                reverse(s0, n)
                continue
            nsub = math.ceil(n / self.K2)
            fwd.set_segment(self.rdesc, [None] * 6, [None] * 3, 0, 0)
            for jj in range(nsub):  # sub-checkpoints of this segment
                for q, t in enumerate(fwd.state_tensors()):
                    self.ckpt2[jj, q].copy_(t)
                if jj < nsub - 1:
                    fwd.run(self.rdesc, False, s0 + jj * self.K2, self.K2)
            for jj in reversed(range(nsub)):
                for q, t in enumerate(fwd.state_tensors()):
                    t.copy_(self.ckpt2[jj, q])
                reverse(s0 + jj * self.K2, min(self.K2, n - jj * self.K2))
        fwd.set_segment(self.rdesc, [None] * 6, [None] * 3, 0, 0)
        return tuple(k)

    def _adjoint_batch(self):
        """The adjoint batch and its receiver injection lists (on the
        device), made by the first backward and kept, so that later
        backwards make no host-to-device copy (and can be captured in a
        CUDA graph)."""
        if self._adj is None:
            adj = ShotBatch(self.model, self.nshots, self.nt, self.rec_id)
            inj = (engine.upload_lists(adjoint_injection_lists(self.nshots, self.rec_id), self.model.device)
                   if len(self.rec_id) else None)
            self._adj = (adj, inj)
        return self._adj

    def _backward_overlapped(self, adj: ShotBatch, adesc) -> None:
        """The levels = 1 backward with the recomputation one segment ahead
        on a second stream: segment s-1 is recomputed into one store buffer
        while the transposes of segment s read the other; a buffer is
        refilled only after the transposes that read it (CUDA events).  The
        recomputing stream has the higher priority, so its CTAs are placed
        first and the transposed steps fill the SMs around them (measured
        at 512 x 512 x 32 shots: 56.1 against 55.7 Gcell/s with equal
        priorities and 54.5 the other way round)."""
        fwd = self.fwd
        main = torch.cuda.current_stream() if adj.stream is None else adj.stream
        if self._side is None:
            self._side = torch.cuda.Stream(device=self.model.device, priority=torch.cuda.Stream.priority_range()[1])
        side = self._side
        side.wait_stream(main)  # the forward sweep and the trace sums
        bufs = ((self.seg_e, self.seg_ds), (self.seg_e2, self.seg_ds2))
        freed = [None, None]  # per buffer: event after the last transposes that read it

        def recompute(s):
            j = s % 2
            s0, n = s * self.K, min(self.K, self.t0 - s * self.K)
            with torch.cuda.stream(side):
                if freed[j] is not None:
                    side.wait_event(freed[j])
                for q, t in enumerate(fwd.state_tensors()):
                    t.copy_(self.ckpt[s, q])
                fwd.set_segment(self.rdesc, bufs[j][0], bufs[j][1], s0, n)
                fwd.run(self.rdesc, False, s0, n)
                ev = torch.cuda.Event()
                ev.record(side)
            return ev

        saved = fwd.stream
        fwd.stream = side
        self.rdesc.ctas_per_sm = self.overlap_ctas
        self.rdesc.step_overlap = 0  # shares the SMs with the transposed steps
        try:
            ready = recompute(self.nseg - 1)
            if self.tail:
                adj.set_segment(adesc, self.tail_e, self.tail_ds, self.t0, self.tail)
                adj.run_transposed(adesc, self.nt, self.tail)
            for s in reversed(range(self.nseg)):
                main.wait_event(ready)
                ready = recompute(s - 1) if s > 0 else None
                j = s % 2
                s0, n = s * self.K, min(self.K, self.t0 - s * self.K)
                adj.set_segment(adesc, bufs[j][0], bufs[j][1], s0, n)
                adj.run_transposed(adesc, s0 + n, n)
                freed[j] = torch.cuda.Event()
                freed[j].record(main)
            main.wait_stream(side)
        finally:
            fwd.stream = saved
            self.rdesc.ctas_per_sm = fwd.ctas_per_sm
            self.rdesc.step_overlap = self.step_overlap
            fwd.set_segment(self.rdesc, [None] * 6, [None] * 3, 0, 0)


def _pad(t: torch.Tensor, grid: Grid) -> torch.Tensor:
    out = torch.zeros((grid.nx, grid.pitch), dtype=torch.float32, device=t.device)
    out[:, : grid.nz] = t.reshape(grid.nx, grid.nz)
    return out


class GradientGraph:
    """One exact gradient -- the checkpointed forward sweep, the caller's
    misfit step and the backward -- captured in two CUDA graphs that share
    one memory pool, so that a gradient of all shots of the batch is two
    launches from the host (its thousands of step kernels, copies and the
    overlapped backward's two streams become graph nodes; the
    programmatic-dependent-launch edges of the forward sweep are kept).
    The split lets a caller upload the observed traces that the misfit step
    reads while the forward sweep runs.

    ``between(traces)`` enqueues the misfit work on the current stream and
    returns (trace gradients per component slot, extra outputs); it must
    neither synchronise nor copy from host memory.  Construction runs one
    eager gradient first (it makes the adjoint batch and fills the
    library's launch caches; ``warm_up=False`` skips it when ``ea`` has
    just computed one) and then captures one, on the model's stream when it
    has one.  ``replay()`` (or ``replay_forward()`` then
    ``replay_backward()``) computes the gradient for the model's current
    values (update the model tensors in place between replays) on the
    current stream and returns (traces, extra, kernels): tensors owned by
    the graphs that the next replay overwrites.  The values are those of
    the eager ExactAdjoint.forward / backward, bit for bit.  ``launches`` is
    the number of library kernels one gradient runs."""

    def __init__(self, ea: ExactAdjoint, between, warm_up: bool = True):
        self.ea = ea
        if ea.step_events is not None:
            raise ValueError("GradientGraph: step events cannot be recorded inside a graph")
        dev = ea.model.device
        stream = ea.model.stream  # the batches' stream (None: the current one)
        if warm_up:
            main = torch.cuda.current_stream(dev)
            warm = stream if stream is not None else torch.cuda.Stream(device=dev)
            warm.wait_stream(main)
            with torch.cuda.stream(warm):
                g, _ = between(ea.forward())
                ea.backward(g)
            main.wait_stream(warm)
        lib = engine._lib.load()
        n0 = lib.fwi_launch_count()
        self.forward_graph, self.backward_graph = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        # thread_local: host threads that stage data meanwhile do not void the capture
        with torch.cuda.graph(self.forward_graph, stream=stream, capture_error_mode="thread_local"):
            self.traces = ea.forward()
        with torch.cuda.graph(self.backward_graph, pool=self.forward_graph.pool(), stream=stream,
                              capture_error_mode="thread_local"):
            g, self.extra = between(self.traces)
            self.kernels = ea.backward(g)
        self.launches = lib.fwi_launch_count() - n0
        self.illum = ea.illum

    def replay_forward(self):
        """The forward sweep; returns the traces."""
        self.forward_graph.replay()
        return self.traces

    def replay_backward(self):
        """The misfit step and the backward of the last forward sweep;
        returns (extra, kernels)."""
        self.backward_graph.replay()
        return self.extra, self.kernels

    def replay(self):
        self.replay_forward()
        self.replay_backward()
        return self.traces, self.extra, self.kernels


class Seismograms(torch.autograd.Function):
    """(lam, mu, rho) -> receiver traces, differentiable.

    Inputs are float32 CUDA tensors of shape [nx, nz] (the reference's cell
    order).  ``setup`` is an :class:`AcquisitionSetup`.  Output: traces
    [ncomp, nshots, nrec, nt] (SH: the y component; P-SV: x then z).
    Gradients are the exact discrete adjoint (FP64 accumulation)."""

    @staticmethod
    def forward(ctx, lam, mu, rho, setup):
        g = setup.grid
        m = DeviceModel(g, setup.mode, setup.dt, lam.device)
        m.lam.copy_(_pad(lam.detach(), g))
        m.mu.copy_(_pad(mu.detach(), g))
        m.rho.copy_(_pad(rho.detach(), g))
        w, a, l, r, b, t = setup.absorb
        lib = engine._lib.load()
        engine.check(lib.fwi_set_bound(engine.ptr(m.bound), g.nx, g.nz, g.pitch, int(w), float(a), int(l), int(r),
                                       int(b), int(t), engine.stream_handle(None)), "fwi_set_bound")
        m.prepare()
        # the divergence stores only where rho needs a gradient
        ea = ExactAdjoint(m, setup.nt, setup.src_id, setup.isrc_of_shot, setup.nshots, setup.stf, setup.rec_id,
                          segment=setup.segment, density=bool(ctx.needs_input_grad[2]))
        tr = ea.forward()
        comps = [c for c in range(3) if tr[c] is not None]
        ctx.ea, ctx.comps, ctx.setup = ea, comps, setup
        ctx.save_for_backward(rho)
        return torch.stack([tr[c] for c in comps])

    @staticmethod
    def backward(ctx, grad):
        (rho,) = ctx.saved_tensors
        g = ctx.setup.grid
        gt = [None, None, None]
        for i, c in enumerate(ctx.comps):
            gt[c] = grad[i]
        k_lam, k_mu, k_buo = ctx.ea.backward(gt)
        engine.check_device(None, "Seismograms.backward")
        nz = g.nz
        dlam = k_lam[:, :nz].reshape(g.nx, nz)
        dmu = k_mu[:, :nz].reshape(g.nx, nz)
        # buo = dt/rho rounded to float32 -> dL/drho = -dL/dbuo * dt / rho^2
        drho = None if k_buo is None else (-k_buo[:, :nz].reshape(g.nx, nz) * ctx.setup.dt / rho.double() ** 2).float()
        ctx.ea = None
        return dlam.float(), dmu.float(), drho, None


class AcquisitionSetup:
    """Everything of a batched simulation except the model: grid, time axis,
    sources (positions and Ricker parameters), receivers and sponge."""

    def __init__(self, mode: str, grid: Grid, dt: float, nt: int, src: np.ndarray, rec: np.ndarray, absorb,
                 combine_sources: bool = False, segment: int | None = None, device="cuda"):
        from ._lib import MODES
        self.mode = MODES[mode]
        self.grid, self.dt, self.nt = grid, float(dt), int(nt)
        self.absorb = absorb
        self.src_id = engine.point_ids(np.asarray(src, np.float64), np.float32(grid.dx), np.float32(grid.dz), grid.nz)
        self.rec_id = engine.point_ids(np.asarray(rec, np.float64), np.float32(grid.dx), np.float32(grid.dz), grid.nz)
        self.nshots = 1 if combine_sources else len(self.src_id)
        self.isrc_of_shot = (lambda s: -1) if combine_sources else (lambda s: s)
        self.stf, self._par = engine.ricker_stf(np.asarray(src, np.float64), self.nt, self.dt, device)
        self.segment = segment


def hann_taper(nt: int, dt: float) -> np.ndarray:
    """The misfit's time taper (waveform.py:11-21), float64."""
    t_end = (nt - 1) * dt
    tw = t_end / 10
    t_min, t_max = tw, t_end - tw
    w = np.ones(nt)
    for it in range(nt):
        t = it * dt
        if t <= t_min:
            w[it] = 0.5 + 0.5 * math.cos(math.pi * (t_min - t) / tw)
        elif t >= t_max:
            w[it] = 0.5 + 0.5 * math.cos(math.pi * (t_max - t) / tw)
    return w


def waveform_misfit(traces: torch.Tensor, data: torch.Tensor, dt: float) -> torch.Tensor:
    """chi = sum taper^2 (syn - data)^2 in FP64 -- the objective whose negative
    derivative is the reference's adjoint source 2 taper^2 (d - s)
    (waveform.py:24-25)."""
    w = torch.as_tensor(hann_taper(traces.shape[-1], dt), device=traces.device)
    r = (traces.double() - data.double()) * w
    return (r * r).sum()


def vps_to_lame(vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor):
    """vps2lm (fd2d.py:21-33) in differentiable torch ops (vp > vs assumed)."""
    return rho * (vp * vp - 2 * vs * vs), rho * vs * vs
