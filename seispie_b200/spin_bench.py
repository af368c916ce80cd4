"""Micropolar-spin forward + exact adjoint with two-level checkpointing.

    python -m seispie_b200.spin_bench [--nx 4096 --nz 2048 --shots 8 --nt 8000 --batch 4]

The spin medium of the reference's example (examples/spin/generate_model.py:
rho 2700, lambda = mu = 8.1e9, nu 1.005e9, j 2700, mu_c 1.5e8, nu_c 3e8;
dx = dz = 1 m as examples/spin/config.ini) with a +-5 %
checkerboard in mu (64-cell squares) as the true model and the homogeneous
medium as the current one.  dt defaults to 1.5e-4 s: the example's 2e-4 s
is 0.99 of the 4th-order staggered-grid stability limit dx / (vp sqrt(2)
(9/8 + 1/24)) for vp = 3000 m/s, and the stiffer squares of the true model
(vp 3050 m/s) exceed it.  Ricker sources (f0 = 100 Hz) along a line at
z = 10 cells, receivers every 8 cells at z = 12.  Observed data are
generated untimed; the timed part is one gradient of all shots in batches of
`--batch`: forward with level-1 checkpoints, trace gradients of the L2
misfit, two-level checkpointed backward with the exact transposed spin step.
Prints one JSON line: useful cell-updates per second (2 x shots x cells x nt
/ device time), per-phase times, the checkpoint layout and the device memory
held by one batch.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--nz", type=int, default=2048)
    ap.add_argument("--shots", type=int, default=8)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--nt", type=int, default=8000)
    ap.add_argument("--nrec", type=int, default=0, help="default: one every 8 cells in x")
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--dt", type=float, default=1.5e-4)
    a = ap.parse_args(argv)
    from . import engine
    from .adjoint import ExactAdjoint, two_level_segments
    from .engine import Grid, build_model
    dev = torch.device("cuda")
    nx, nz, h, dt, nt = a.nx, a.nz, 1.0, a.dt, a.nt
    npt = nx * nz
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    board = np.where(((i // 64) + (j // 64)) % 2 == 0, 1.0, -1.0).ravel()
    base = dict(rho=np.full(npt, 2700.0), lam=np.full(npt, 8.1e9), mu=np.full(npt, 8.1e9), nu=np.full(npt, 1.005e9),
                j=np.full(npt, 2700.0), mu_c=np.full(npt, 1.5e8), nu_c=np.full(npt, 3.0e8))
    true = dict(base, mu=8.1e9 * (1 + 0.05 * board))
    grid = Grid(nx, nz, h, h)
    absorb = (20, 0.015, 1, 1, 1, 0)
    nrec = a.nrec or nx // 8
    src = np.array([[(s + 0.5) * nx / a.shots * h, 10 * h, 0, 100.0, 0.012, 0.0, 1e10] for s in range(a.shots)])
    rec = np.array([[(r + 0.5) * nx / nrec * h, 12 * h] for r in range(nrec)])
    sid = engine.point_ids(src, np.float32(h), np.float32(h), nz)
    rid = engine.point_ids(rec, np.float32(h), np.float32(h), nz)
    stf, _ = engine.ricker_stf(src, nt, dt, dev)
    m_true = build_model("spin", grid, dt, true, absorb, dev)
    m_cur = build_model("spin", grid, dt, base, absorb, dev)
    k1, k2 = two_level_segments(nt, 2)
    batches = [list(range(s, min(s + a.batch, a.shots))) for s in range(0, a.shots, a.batch)]
    # observed data (untimed)
    data = {}
    for b in batches:
        ea = ExactAdjoint(m_true, nt, sid, lambda s, b=b: b[s], len(b), stf, rid, levels=a.levels)
        tr = ea.forward()
        data[b[0]] = [tr[c].clone() if c != 1 else None for c in range(3)]
        del ea
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    t_fwd = t_adj = 0.0
    misfit = 0.0
    ev[0].record()
    t0 = time.time()
    for b in batches:
        n = len(b)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ea = ExactAdjoint(m_cur, nt, sid, lambda s, b=b: b[s], n, stf, rid, levels=a.levels)
        e[0].record()
        tr = ea.forward()
        e[1].record()
        g = [None, None, None]
        for c in (0, 2):
            g[c] = torch.empty(n * nrec * nt, dtype=torch.float32, device=dev)
            misfit += float(engine.misfit_tracegrad(data[b[0]][c].reshape(-1), tr[c].reshape(-1).contiguous(), g[c],
                                                    n, nrec, nt, dt).sum().item())
            g[c] = g[c].view(n, nrec, nt)
        ks = ea.backward(g)
        e[2].record()
        torch.cuda.synchronize()
        t_fwd += e[0].elapsed_time(e[1]) * 1e-3
        t_adj += e[1].elapsed_time(e[2]) * 1e-3
        del ea, ks
    ev[1].record()
    torch.cuda.synchronize()
    total = ev[0].elapsed_time(ev[1]) * 1e-3
    cells = 2.0 * a.shots * npt * nt
    print(json.dumps({"workload": "spin_gradient_%dx%d_shots%d_nt%d" % (nx, nz, a.shots, nt),
                      "value": cells / total / 1e9, "unit": "Gcell-updates/s (useful: forward + adjoint)",
                      "seconds": total, "forward_s": t_fwd, "backward_s": t_adj, "wall_s": time.time() - t0,
                      "batches": len(batches), "batch_shots": a.batch, "levels": a.levels,
                      "segments": [k1, k2] if a.levels == 2 else None,
                      "peak_device_gb": torch.cuda.max_memory_allocated() / 1e9, "misfit": misfit}))


if __name__ == "__main__":
    main()
