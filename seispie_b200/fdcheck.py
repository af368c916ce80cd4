"""Finite-difference check of the exact gradient at full scale.

    python -m seispie_b200.fdcheck [--nx 512 --nz 512 --shots 32 --nrec 256 --nt 4000 --cells 16 --h 0.02]

P-SV gradient configuration: 512 x 512, h = 10 m, vp 3000 / vs 1732 / rho
2600 background with a +-5 % vs checkerboard (32 x 32 squares) for the data,
32 Ricker sources (8 Hz) at z = 10 cells, 256 receivers at z = 12 cells,
dt = 1e-3, nt = 4000.  The gradient of chi = sum taper^2 (s - d)^2 with
respect to mu comes from the autograd.Function (exact discrete adjoint with
checkpointing); each of --cells random interior cells is then perturbed by
+-h*mu and chi re-evaluated with the GPU forward (central difference).
Prints one JSON line with the per-cell relative errors.  The FP64 oracle
checks of the same gradient at small sizes live in tests/test_gpu_adjoint.py.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--nz", type=int, default=512)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--nrec", type=int, default=256)
    ap.add_argument("--nt", type=int, default=4000)
    ap.add_argument("--cells", type=int, default=16)
    ap.add_argument("--h", type=float, default=0.02)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    from .adjoint import AcquisitionSetup, Seismograms, waveform_misfit
    from .engine import Grid

    nx, nz, h = a.nx, a.nz, 10.0
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    board = np.where(((i // 32) + (j // 32)) % 2 == 0, 1.0, -1.0)
    rho = torch.full((nx, nz), 2600.0, device="cuda")
    vp = torch.full((nx, nz), 3000.0, device="cuda")
    vs0 = torch.full((nx, nz), 1732.0, device="cuda")
    vs_true = torch.as_tensor((1732.0 * (1 + 0.05 * board)).astype(np.float32), device="cuda")
    src = np.array([[(s + 0.5) * nx / a.shots * h, 10 * h, 0, 8.0, 0.15, 0.0, 1e10] for s in range(a.shots)])
    rec = np.array([[(r + 0.5) * nx / a.nrec * h, 12 * h] for r in range(a.nrec)])
    setup = AcquisitionSetup("psv", Grid(nx, nz, h, h), 1e-3, a.nt, src, rec, (20, 0.015, 1, 1, 1, 0))

    def lame(vsx):
        return rho * (vp * vp - 2 * vsx * vsx), rho * vsx * vsx

    with torch.no_grad():
        lt, mt = lame(vs_true)
        data = Seismograms.apply(lt, mt, rho, setup).detach()
    lam, mu = lame(vs0)
    mu = mu.clone().requires_grad_(True)
    t0 = time.time()
    chi = waveform_misfit(Seismograms.apply(lam, mu, rho, setup), data, setup.dt)
    chi.backward()
    torch.cuda.synchronize()
    t_grad = time.time() - t0
    g = mu.grad.double().cpu().numpy()
    rng = np.random.default_rng(a.seed)
    # cells spread over the illuminated part of the model (below the sources, inside the sponge)
    cells = [(int(rng.integers(40, nx - 40)), int(rng.integers(20, nz // 2))) for _ in range(a.cells)]
    out = []
    with torch.no_grad():
        for (ci, cj) in cells:
            dm = a.h * float(mu[ci, cj])
            vals = []
            for sgn in (1.0, -1.0):
                m2 = mu.detach().clone()
                m2[ci, cj] += sgn * dm
                vals.append(float(waveform_misfit(Seismograms.apply(lam, m2, rho, setup), data, setup.dt)))
            fd = (vals[0] - vals[1]) / (2 * dm)
            out.append(dict(cell=[ci, cj], grad=float(g[ci, cj]), fd=fd,
                            rel_err=abs(g[ci, cj] - fd) / max(abs(fd), 1e-300)))
    line = {"workload": "psv_fd_check_%dx%d_shots%d_nt%d" % (nx, nz, a.shots, a.nt), "h_rel": a.h,
            "chi": float(chi), "gradient_seconds": t_grad, "segment": None,
            "median_rel_err": float(np.median([o["rel_err"] for o in out])),
            "max_rel_err": float(max(o["rel_err"] for o in out)), "cells": out}
    print(json.dumps(line))
    return line


if __name__ == "__main__":
    main()
