#!/usr/bin/env python
"""Benchmark of the FWI hot path: batched P-SV forward + adjoint gradient.

Workload (the P-SV gradient configuration): 512 x 512 grid, h = 10 m,
vp 3000 / vs 1732 (+-5 % checkerboard in 32 x 32-cell squares for the true
model, homogeneous start) / rho 2600, 32 Ricker sources (f0 = 8 Hz) evenly
spaced at z = 10 cells, 256 receivers at z = 12 cells, dt = 1e-3 s,
nt = 4000, 20-cell sponge on the left, right and bottom, adjoint interval 10,
smoothing sigma 4.  Observed data come from the checkerboard model (computed
once, untimed).  One step = one gradient of all shots: batched forward with
checkpoints (row-marching step kernel, no displacement field), misfit and
trace gradients, exact discrete adjoint (checkpointed recomputation +
transposed steps with the lambda / mu terms), Gaussian smoothing
(``--gradient reference``: forward with snapshots and the
snapshot-correlation adjoint instead).  Cell-updates per step =
shots * 512 * 512 * 4000 * 2 (forward and adjoint counted separately;
recomputed forward steps are not counted).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--shard]
                    [--density 0|1] [--overlap 0|1] [--step-overlap 0|1] [--profile-case]

The gradient is the λ and μ kernels (the reference's gradient is μ); --density 1 adds the ρ
kernel, whose divergence stores shorten the stored tail.  --overlap 0 runs the backward on one
stream (recomputation and transposed steps in turn).  --step-overlap 0 launches the steps of the
forward sweep without programmatic dependent launch.

On N GPUs (torchrun, one rank per GPU) every rank owns a contiguous block of
the shots and the ranks sum the FP64 mu kernel and the misfit with one
all-reduce before the smoothing, as the reference sums before it smooths
(solver.py:375-396).  By default each rank has 32 shots (the survey grows
with N: weak scaling); ``--shard`` splits the 32 shots over the ranks
(strong scaling).

Prints one JSON line (rank 0).  ``value`` is measured with every input in HBM,
on the exact gradient captured once in a CUDA graph and replayed per step
(seispie_b200.adjoint.GradientGraph: two host launches per gradient; the
all-reduce and the smoothing run eagerly); ``eager`` holds the same gradient
launched step by step, whose CUDA events time the roofline's kernel
(``--graph 0`` makes the step-by-step gradient the value);
``e2e`` through the plugin API (seispie_b200.solver.b200.compute_gradient)
with the observed traces in host memory, their upload and the gradient's
download inside the timed region.  ``roofline`` is the row-marching step
kernel's (CUDA events around its launches inside the eager timed region);
``gradient_roofline`` the whole gradient's useful cell-update rate in the
same bytes.  ``--impl reference`` times the CPU restatement of the
reference's arithmetic (oracle/, float32, all host threads) on a bounded
sample of the same workload, and reports beside it the unmodified reference
timed under Numba's CUDA simulator (oracle/reference_cudasim.json).
"""
from __future__ import annotations

import argparse
import contextlib
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s (P-SV forward+adjoint gradient, batched shots)"
UNIT = "Gcell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--nz", type=int, default=512)
    ap.add_argument("--nt", type=int, default=4000)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--nrec", type=int, default=256)
    ap.add_argument("--sae", type=int, default=10)
    ap.add_argument("--sigma", type=int, default=4)
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    ap.add_argument("--profile-case", action="store_true",
                    help="only 20 forward steps and one gradient of --nt steps (for ncu captures of the kernels)")
    ap.add_argument("--autotune", action="store_true", help="time every tile variant and report the best")
    ap.add_argument("--overlap", type=int, default=1, choices=[0, 1],
                    help="1: recompute segment s-1 on a second stream while segment s is transposed")
    ap.add_argument("--tail-budget", type=float, default=0.93,
                    help="fraction of the free HBM the exact gradient's buffers and stored tail may take")
    ap.add_argument("--density", type=int, default=0, choices=[0, 1],
                    help="1: also the density kernel (stores the divergence per step); 0: lambda and mu kernels")
    ap.add_argument("--overlap-ctas", type=int, default=0,
                    help="with --overlap: resident CTAs per SM of the recomputing step (0: all that fit)")
    ap.add_argument("--step-overlap", type=int, default=1, choices=[0, 1],
                    help="1: programmatic dependent launch between the steps of a time loop that has the GPU to "
                         "itself (the forward sweep; the overlapped backward's streams never use it); 0: none")
    ap.add_argument("--graph", type=int, default=1, choices=[0, 1],
                    help="1: value is the exact gradient captured in CUDA graphs (forward sweep; misfit and "
                         "backward) replayed as two launches per gradient (the step-by-step gradients that carry the "
                         "roofline's events are reported under 'eager'); 0: value is the step-by-step gradient")
    ap.add_argument("--shard", action="store_true",
                    help="split the --shots shots over the ranks (strong scaling) instead of --shots per rank")
    ap.add_argument("--gradient", default="exact", choices=["exact", "reference"],
                    help="exact: discrete adjoint with checkpointing (the solver's P-SV gradient); "
                         "reference: snapshot-correlation adjoint of the reference's algorithm")
    return ap.parse_args()


# ------------------------------------------------------------------ workload

def total_shots(a, world):
    """Shots of the whole job: --shots per rank, or --shots split over the
    ranks with --shard."""
    return a.shots if a.shard else a.shots * world


def workload(a, nshots=None):
    nshots = a.shots if nshots is None else nshots
    nx, nz, h = a.nx, a.nz, 10.0
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    sign = np.where(((i // 32) + (j // 32)) % 2 == 0, 1.0, -1.0)
    vs_true = (1732.0 * (1 + 0.05 * sign)).ravel().astype(np.float32)
    n = nx * nz
    vp = np.full(n, 3000.0, np.float32)
    rho = np.full(n, 2600.0, np.float32)
    vs_init = np.full(n, 1732.0, np.float32)
    f0 = 8.0
    src = np.array([[(s + 0.5) * nx / nshots * h, 10 * h, 0, f0, 1.2 / f0, 0.0, 1e10] for s in range(nshots)])
    rec = np.array([[(r + 0.5) * nx / a.nrec * h, 12 * h] for r in range(a.nrec)])
    return dict(nx=nx, nz=nz, h=h, dt=1e-3, vp=vp, rho=rho, vs_true=vs_true, vs_init=vs_init, src=src, rec=rec,
                absorb=(20, 0.015, 1, 1, 1, 0))


def config_of(a, w, extra=None, world=1):
    ns = total_shots(a, world)
    c = {"workload": "psv_gradient_%dx%d_shots%d_rec%d_nt%d" % (a.nx, a.nz, a.shots, a.nrec, a.nt),
         "grid": [a.nx, a.nz], "shots": ns, "shots_per_rank": ns // world, "receivers": a.nrec, "nt": a.nt,
         "adjoint_interval": a.sae, "smooth_sigma": a.sigma, "cells_per_step": 2 * ns * a.nx * a.nz * a.nt,
         "l2": "inputs larger than L2 (each wavefield field of 32 shots is 32 MiB, the state 5 fields, the "
               "checkpoints and stored steps ~150 GB: far above the 126 MB L2); no flush",
         "parallelism": "shots (contiguous blocks per rank, one FP64 all-reduce per gradient)"
                        if world > 1 else "shots", "gradient": a.gradient,
         "step_overlap": bool(getattr(a, "step_overlap", 1)) and getattr(a, "impl", "b200") == "b200",
         "cuda_graph": bool(getattr(a, "graph", 0)) and a.gradient == "exact" and getattr(a, "impl", "b200") == "b200"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
        return False

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                               r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ reference arm

def cpu_sample(a, w, seconds):
    """Time the oracle's float32 restatement of the reference (forward and
    adjoint of one shot, all host threads) for about ``seconds``.  The
    adjoint timed is the reference's snapshot-correlation adjoint
    (solver.py:290-321, extended to P-SV), which does less work than the
    exact adjoint with recomputation the GPU runs.  Returns (cell-updates/s,
    sample dict, threads)."""
    from oracle.oracle import Oracle, point_ids, source_time_functions
    o = Oracle("f32")
    nx, nz, h, dt = w["nx"], w["nz"], w["h"], w["dt"]
    lam, mu = o.vps2lm(w["vp"], w["vs_init"], w["rho"])
    bound = o.set_bound(nx, nz, *w["absorb"])
    p = dict(rho=w["rho"], lam=lam, mu=mu, bound=bound)
    sid = point_ids(w["src"], np.float32(h), np.float32(h), nz)
    rid = point_ids(w["rec"], np.float32(h), np.float32(h), nz)
    # calibrate on a short run, then size the sample to ~seconds
    nt0 = 20
    stf = source_time_functions(w["src"][:1], nt0, dt)
    t = time.perf_counter()
    o.forward("psv", nx, nz, h, h, dt, nt0, p, sid[:1], stf, 0, rid)
    rate0 = nx * nz * nt0 / (time.perf_counter() - t)
    nt = int(max(2 * a.sae, min(a.nt, seconds * rate0 / 2 / nx / nz)))
    nt -= nt % a.sae
    stf = source_time_functions(w["src"][:1], nt, dt)
    t = time.perf_counter()
    obs, _, sn = o.forward("psv", nx, nz, h, h, dt, nt, p, sid[:1], stf, 0, rid, sae=a.sae, nsa=nt // a.sae,
                           snapshots=True)
    ad = np.random.default_rng(0).standard_normal(len(rid) * nt).astype(np.float32)
    k = [np.zeros(nx * nz, np.float32) for _ in range(3)]
    o.adjoint_psv(nx, nz, h, h, dt, nt, p, rid, ad, ad, a.sae, sn, k[0], k[1], k[2])
    el = time.perf_counter() - t
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cells = 2 * nx * nz * nt
    sample = {"what": "1 shot of %dx%d, nt=%d: forward + snapshot-correlation adjoint of the float32 oracle "
                      "(the reference's arithmetic)" % (nx, nz, nt),
              "shots": 1, "nt": nt, "cell_updates": cells, "seconds": el}
    return cells / el / 1e9, sample, threads


def reference_cudasim():
    """The unmodified reference timed under Numba's CUDA simulator by
    oracle/time_reference.py (measured where that script ran, recorded in
    oracle/reference_cudasim.json), or None."""
    try:
        rec = json.load(open(os.path.join(ROOT, "oracle", "reference_cudasim.json")))
    except Exception:
        return None
    c = rec["cases"]
    return {"value": c["psv_forward"]["cell_updates_per_s"] / 1e9, "unit": UNIT, "cores": rec["cores_used"],
            "kind": "reference", "nproc": rec["nproc"],
            "sample": rec["what"] + " (P-SV forward; the reference's P-SV adjoint cannot run; SH gradient "
                                    "%.3g cell-updates/s)" % c["sh_gradient"]["cell_updates_per_s"],
            "measured": "build container (numba %s), not the GPU host: the reference's Python source does not "
                        "travel to the GPU box" % rec["numba"]}


def run_reference(a):
    """Reference arm: the CPU restatement of the reference's arithmetic on a
    bounded sample of the workload per step; ms_per_step is the sample's own
    time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(a)
    vals, secs = [], []
    sample = threads = None
    for s in range(a.warmup + a.steps):
        v, sample, threads = cpu_sample(a, w, a.cpu_seconds / max(1, a.steps))
        if s >= a.warmup:
            vals.append(v)
            secs.append(sample["seconds"])
    v = statistics.median(vals)
    cfg = config_of(a, w)
    cfg["cells_per_step"] = sample["cell_updates"]  # each step is one bounded sample
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": statistics.median(secs) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "reference_cudasim": reference_cudasim(),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm

def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from seispie_b200 import _lib, engine
    from seispie_b200.engine import Grid, ShotBatch, adjoint_injection_lists, build_model, injection_lists
    from seispie_b200.parallel import shard

    lib = _lib.load()
    ntot = total_shots(a, world)
    mine = list(shard(ntot, rank, world))  # this rank's contiguous block of shots
    w = workload(a, ntot)
    nx, nz, h, dt, nt = w["nx"], w["nz"], w["h"], w["dt"], a.nt
    sid = engine.point_ids(w["src"], np.float32(h), np.float32(h), nz)
    rid = engine.point_ids(w["rec"], np.float32(h), np.float32(h), nz)
    grid = Grid(nx, nz, float(np.float32(h)), float(np.float32(h)))
    m_true = build_model("psv", grid, dt, dict(vp=w["vp"], vs=w["vs_true"], rho=w["rho"]), w["absorb"], dev)
    m_init = build_model("psv", grid, dt, dict(vp=w["vp"], vs=w["vs_init"], rho=w["rho"]), w["absorb"], dev)
    stf, _ = engine.ricker_stf(w["src"], nt, dt, dev)
    nshots = len(mine)
    inj = injection_lists(nshots, sid, lambda s: mine[s])

    if a.profile_case:
        # 20 forward steps of the batch, then one exact gradient of nt steps (all of them stored
        # from the forward sweep): the row-marching step and the transposed step at full size
        b = ShotBatch(m_init, nshots, nt, rid, tile=a.tile)
        d = b.desc(inj=inj, stf=stf)
        b.clear()
        b.run(d, False, 0, min(nt, 20))
        from seispie_b200.adjoint import ExactAdjoint
        ea = ExactAdjoint(m_init, nt, sid, lambda s: mine[s], nshots, stf, rid, tail_memory=1e30,
                          density=bool(a.density))
        ea.forward()
        gen = torch.Generator(device=dev).manual_seed(0)
        g = [torch.randn((nshots, a.nrec, nt), generator=gen, device=dev) if c != 1 else None for c in range(3)]
        ea.backward(g)
        torch.cuda.synchronize()
        engine.check_device(None, "profile case")
        print(json.dumps({"profile_case": True, "forward_steps": min(nt, 20), "gradient_steps": nt}))
        return

    # observed data from the checkerboard model (untimed)
    bt = ShotBatch(m_true, nshots, nt, rid, tile=a.tile)
    bt.clear()
    bt.run(bt.desc(inj=inj, stf=stf), False, 0, nt)
    data = [bt.obs[0].clone(), None, bt.obs[2].clone()]
    del bt

    stream = torch.cuda.current_stream()
    ev = {}

    def reduce_and_smooth(mis, k_mu):
        """Sum the ranks' FP64 mu kernels and misfits, then smooth (the
        reference's order, solver.py:375-396)."""
        m = torch.stack([x.sum() for x in mis]).sum()
        if world > 1:
            dist.all_reduce(k_mu)
            dist.all_reduce(m)
        return m, engine.smooth(k_mu, m_init.grid, a.sigma)

    if a.gradient == "exact":
        # exact discrete adjoint with checkpointed recomputation (the P-SV gradient of the solver)
        from seispie_b200._lib import FWI_PSV
        from seispie_b200.adjoint import ExactAdjoint, max_tail_bytes
        # per-step stores of the last steps kept from the forward sweep: the longest tail that fits
        # --tail-budget of the free HBM with the checkpoints, segment stores, wavefields and traces
        free, _ = torch.cuda.mem_get_info(dev)
        # the mu kernel (the reference's) and the lambda kernel, no density kernel: no divergence stores
        tail = max_tail_bytes(nt, FWI_PSV, nshots, m_init.grid, a.tail_budget * free, a.nrec,
                              overlap=bool(a.overlap), density=bool(a.density))
        ea = ExactAdjoint(m_init, nt, sid, lambda s: mine[s], nshots, stf, rid, tile=a.tile, tail_memory=tail,
                          overlap=bool(a.overlap), overlap_ctas=a.overlap_ctas, density=bool(a.density),
                          step_overlap=bool(a.step_overlap))
        checkpointing = {"segment": ea.K, "checkpoints": ea.nseg, "stored_tail_steps": ea.tail,
                         "overlap": ea.overlap, "overlap_ctas": ea.overlap_ctas}
        kernels = ["lam", "mu"] + (["rho"] if ea.density else [])
        grads = [torch.empty((nshots, a.nrec, nt), dtype=torch.float32, device=dev) if c != 1 else None
                 for c in range(3)]
        b = ea.fwd
        fwd = ea.fdesc
        adj = fwd

        def gradient(record=False):
            e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
            ea.step_events = ev.setdefault("steps", []) if record else None
            e0.record(stream)
            tr = ea.forward()
            e1.record(stream)
            mis = [engine.misfit_tracegrad(data[c], tr[c].reshape(-1), grads[c], nshots, a.nrec, nt, dt)
                   for c in (0, 2)]
            e2.record(stream)
            k_lam, k_mu, k_buo = ea.backward(grads)
            e3.record(stream)
            m, g = reduce_and_smooth(mis, k_mu)
            if record:
                ev.setdefault("fwd", []).append((e0, e1))
                ev.setdefault("adj", []).append((e2, e3))
            return m, g
    else:
        nsa = nt // a.sae
        b = ShotBatch(m_init, nshots, nt, rid, sae=a.sae, nsa=nsa, snapshots=True, tile=a.tile)
        k_lam = torch.zeros((nx, m_init.grid.pitch), dtype=torch.float64, device=dev)
        k_mu = torch.zeros_like(k_lam)
        adstf = [torch.empty(nshots * a.nrec * nt, dtype=torch.float32, device=dev) if c != 1 else None
                 for c in range(3)]
        fwd = b.desc(inj=inj, stf=stf)
        adj = b.desc(inj=adjoint_injection_lists(nshots, rid), stf=adstf, record=False,
                     kernels=(k_lam, k_mu, None))

        def gradient(record=False):
            k_lam.zero_()
            k_mu.zero_()
            e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
            b.clear()
            e0.record(stream)
            b.run(fwd, False, 0, nt)
            e1.record(stream)
            mis = [engine.misfit(data[c], b.obs[c], adstf[c], nshots, a.nrec, nt, dt) for c in (0, 2)]
            b.clear()
            e2.record(stream)
            b.run(adj, True, 0, nt)
            e3.record(stream)
            m, g = reduce_and_smooth(mis, k_mu)
            if record:
                ev.setdefault("fwd", []).append((e0, e1))
                ev.setdefault("adj", []).append((e2, e3))
            return m, g

    def tune():
        from seispie_b200.autotune import autotune
        best, times = autotune(m_init, nshots, nt, rid, inj, stf)
        return best, times[best], {_lib.tile_label(t): ms for t, ms in times.items()}

    tuned = None
    if a.autotune:
        tuned = tune()
        b.tile = fwd.tile = adj.tile = tuned[0]

    for _ in range(a.warmup):
        gradient()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = lib.fwi_launch_count()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0.record(stream)
        for _ in range(a.steps):
            mis, g = gradient(record=True)
        t1.record(stream)
        torch.cuda.synchronize()
    launches = lib.fwi_launch_count() - launches0
    ms = t0.elapsed_time(t1) / a.steps
    engine.check_device(stream, "bench")  # no bounded wait gave up in the timed gradients
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        dist.barrier()
    cells = 2 * ntot * nx * nz * nt  # useful cell-updates of the whole job per step
    value = cells / (ms * 1e-3) / 1e9
    misfit_total = float(mis.item())

    # The headline: the same gradient captured in CUDA graphs (forward sweep; misfit and backward) and
    # replayed, two launches per gradient from the host; the eager gradients above, launched step by step,
    # carry the per-launch CUDA events of the roofline.
    eager = None
    if a.gradient == "exact" and a.graph:
        from seispie_b200.adjoint import GradientGraph

        def between(tr):
            return grads, [engine.misfit_tracegrad(data[c], tr[c].reshape(-1), grads[c], nshots, a.nrec, nt, dt)
                           for c in (0, 2)]

        ea.step_events = None  # no per-segment events inside the graph
        gg = GradientGraph(ea, between)
        for _ in range(a.warmup):
            _, gm, gk = gg.replay()
            reduce_and_smooth(gm, gk[1])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        eager = {"value": value, "ms_per_step": ms, "gpu_launches": launches, "clocks": clk.summary(),
                 "note": "the same gradients launched step by step from the host (the roofline's CUDA events)"}
        launches0 = lib.fwi_launch_count()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            g0.record(stream)
            for _ in range(a.steps):
                _, gm, gk = gg.replay()
                gmis, _ = reduce_and_smooth(gm, gk[1])
            g1.record(stream)
            torch.cuda.synchronize()
        # library kernels of the replays (counted once, at capture) plus the smoothing launched eagerly
        launches = gg.launches * a.steps + lib.fwi_launch_count() - launches0
        ms = g0.elapsed_time(g1) / a.steps
        engine.check_device(stream, "bench (graph)")
        eager["graph_misfit_equal"] = float(gmis.item()) == misfit_total  # bit for bit
        if world > 1:
            tt = torch.tensor([ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
            dist.barrier()
        value = cells / (ms * 1e-3) / 1e9
        eager["graph_nodes_library_kernels"] = gg.launches
        del gg

    peak, peak_src = 6650.0, "fallback"
    try:
        pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(pk["hbm_gbs"]), "measured"
    except Exception:
        pass
    fwd_ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev["fwd"])
    adj_ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev["adj"])
    if a.gradient == "exact":
        # the dominant kernel: the row-marching step, timed launch by launch (CUDA events around the plain
        # forward segments of every timed gradient; each segment adds one short trace-conversion launch)
        steps = ev.get("steps", [])
        n_launch = sum(n for _, _, n in steps)
        per_launch_s = sum(e0.elapsed_time(e1) for e0, e1, _ in steps) * 1e-3 / max(1, n_launch)
        # algorithmic bytes: stress (3) and velocity (2) read and written, lam, mu, dt/rho, sponge read
        bytes_per_launch = nshots * nx * nz * (40 + 16)
        kernel = "march_kernel<P-SV> (row-marching step, displacement-free; plain forward launches)"
        traffic_file = "march_kernel_psv_traffic.json"
        if not n_launch:  # every step in the stored tail (short runs): the forward sweep per step
            per_launch_s = fwd_ms * 1e-3 / nt
            kernel = "march_kernel<P-SV> (forward sweep with per-step stores / nt)"
    else:
        per_launch_s = fwd_ms * 1e-3 / nt
        bytes_per_launch = nshots * nx * nz * (72 + 8.0 / a.sae)
        kernel = "step_kernel<P-SV> (tiled, with displacement and snapshots; forward sweep / nt)"
        traffic_file = "step_kernel_psv_traffic.json"
    achieved = bytes_per_launch / per_launch_s / 1e9
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", traffic_file)))
        traffic = prof["dram_bytes_per_launch_full_workload"] * nshots / prof.get("shots", 32)
    except Exception:
        pass
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_src, "kernel": kernel,
            "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_us": per_launch_s * 1e6,
            "launches_timed": n_launch if a.gradient == "exact" else nt,
            "forward_sweep_us_per_step": fwd_ms * 1e3 / nt, "backward_us_per_step": adj_ms * 1e3 / nt}
    # the whole gradient: useful cell-updates per second per GPU times the P-SV algorithmic bytes of a
    # cell-update (72 B), against the same peak
    grad_roof = {"bytes_per_cell_update": 72, "achieved": value / world * 72, "peak": peak, "unit": "GB/s",
                 "frac": value / world * 72 / peak,
                 "basis": "useful forward+adjoint cell-updates (recomputed steps not counted) x 72 B"}

    del b, fwd, adj
    ea = grads = None  # noqa: F841  (release the checkpoint buffers before the e2e run)
    torch.cuda.empty_cache()

    # ----------------------------------------------------------------- e2e
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, w, dev, world, rank, data, ntot)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, sample, threads = cpu_sample(a, w, a.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

    if rank == 0:
        extra = {"tile": _lib.tile_label(b_tile(a, tuned)), "misfit": misfit_total}
        if a.gradient == "exact":
            extra["checkpointing"] = checkpointing
            extra["kernels"] = kernels
            extra["tile"] = "row-marching (displacement-free)"
        if tuned:
            extra["autotune_ms_per_fwd_step"] = tuned[2]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong" if a.shard else "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config_of(a, w, extra, world), "clocks": clk.summary(),
                "gpu_launches": launches, "roofline": roof, "gradient_roofline": grad_roof, "eager": eager, "e2e": e2e,
                "cpu_baseline": cpu, "reference_cudasim": reference_cudasim() if cpu else None, "impl": "b200"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def b_tile(a, tuned):
    return tuned[0] if tuned else a.tile


def run_e2e(a, w, dev, world, rank, data, ntot):
    """compute_gradient() of the b200 plugin with host-resident traces (on N
    ranks through the plugin's own shot sharding and kernel sum)."""
    import torch
    from seispie_b200.solver import b200

    td = tempfile.mkdtemp()
    nx, nz, h = w["nx"], w["nz"], w["h"]
    from seispie_b200.io import write_model
    write_model(td + "/init", nx, nz, h, h, dict(vp=w["vp"], vs=w["vs_init"], rho=w["rho"]))
    np.savetxt(td + "/src.dat", w["src"])
    np.savetxt(td + "/rec.dat", w["rec"])
    os.makedirs(td + "/out", exist_ok=True)
    s = b200()
    s.config = dict(nt=str(a.nt), dt=str(w["dt"]), sh="no", psv="yes", spin="no", abs_left="yes", abs_right="yes",
                    abs_top="no", abs_bottom="yes", abs_width="20", abs_alpha="0.015", save_coordinates="",
                    combine_sources="no", save_snapshot="0", adjoint_interval=str(a.sae), smooth=str(a.sigma),
                    tile=str(a.tile), kernel_rho="yes" if a.density else "no")
    s.path = dict(model_init=td + "/init", model_true=td + "/init", sources=td + "/src.dat",
                  stations=td + "/rec.dat", output=td + "/out")
    if world > 1:
        from seispie_b200.parallel import TorchMPI
        s.mpi = TorchMPI()  # the process group bench.py opened
    else:
        s.mpi = None
    with contextlib.redirect_stdout(io.StringIO()):
        s.setup(None)
        s.import_model(0)
        s.import_sources()
        s.import_stations()
    nloc = len(s._shots())  # this rank's shots, in the order of `data`
    dx = data[0].view(nloc, a.nrec * a.nt).cpu().numpy()
    dz = data[2].view(nloc, a.nrec * a.nt).cpu().numpy()
    s.syn_x = [np.ascontiguousarray(dx[i]) for i in range(nloc)]
    s.syn_z = [np.ascontiguousarray(dz[i]) for i in range(nloc)]
    s.syn_y = []
    h2d = sum(x.nbytes for x in s.syn_x + s.syn_z) * world
    d2h = 2 * nx * nz * 4  # gradient and model returned as float32
    with contextlib.redirect_stdout(io.StringIO()):
        for _ in range(max(1, a.warmup)):
            s.compute_gradient()
        torch.cuda.synchronize()
        if world > 1:
            s.mpi.sync()
        t = time.perf_counter()
        for _ in range(a.steps):
            s.compute_gradient()
        torch.cuda.synchronize()
        el = (time.perf_counter() - t) / a.steps
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([el], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        el = float(tt.item())
    cells = 2 * ntot * nx * nz * a.nt
    return {"value": cells / el / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": el * 1e3, "api": "seispie_b200.solver.b200.compute_gradient"}


if __name__ == "__main__":
    main()
