"""Checkerboard P-SV inversion with the GPU L-BFGS and line search.

    python -m seispie_b200.inversion_bench [--nx 1024 --nz 512 --shots 64 --nt 6000 --niter 20]

Lays out forward / adjoint / inverse directories as the reference's examples
do (config inheritance, model files, sources.dat, stations.dat), then runs the
inversion workflow through seispie_b200.workflow with ``method = b200`` and
``[optimize] method = lbfgs``.  True model: +-8 % checkerboard in vp and vs
(64 x 64-cell squares) on a linear-gradient background; starting model: the
background.  As in the reference the model variable is mu (the gradient is
k_mu), smoothed with sigma = 4 cells.  Prints one JSON line: misfit history
with wall-clock times, seconds per iteration, time to a 90 % misfit drop (if
reached) and the relative L2 error of the final mu against the true mu.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import json
import os
import tempfile
import time

import numpy as np


def write_case(root: str, nx: int, nz: int, shots: int, nrec: int, nt: int, niter: int, sigma: int, sae: int,
               h: float = 10.0, dt: float = 1e-3, square: int = 64, amp: float = 0.08, board=None,
               method: str = "lbfgs", optimize_extra: str = "", perturb: str = "both", invert: str = "mu"):
    """board: perturbation pattern in [-1, 1] ([nx, nz]; default the
    checkerboard of `square`-cell squares); perturb: "both" (vp and vs), "vs"
    (vs only) or "mu" (vs with vp adjusted so that lambda keeps its starting
    value: the model error is then in the inverted parameter mu alone);
    method / optimize_extra: the [optimize] method and further keys
    (lines) of the inversion config; invert: the solver's model variables
    (mu, or vp_vs).  Returns the true (vp, vs, mu)."""
    from .io import write_model
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    vp0 = 3000.0 + 300.0 * (j / (nz - 1) - 0.5)
    vs0 = vp0 / np.sqrt(3.0)
    if board is None:
        board = np.where(((i // square) + (j // square)) % 2 == 0, 1.0, -1.0)
    rho = np.full(nx * nz, 2600.0)
    vs_true = vs0 * (1 + amp * board)
    if perturb == "both":
        vp_true = vp0 * (1 + amp * board)
    elif perturb == "mu":  # lambda of the background kept: only mu differs from the start
        vp_true = np.sqrt(vp0 ** 2 - 2 * vs0 ** 2 + 2 * vs_true ** 2)
    else:
        vp_true = vp0
    true = dict(vp=vp_true.ravel(), vs=vs_true.ravel(), rho=rho)
    init = dict(vp=vp0.ravel(), vs=vs0.ravel(), rho=rho)
    fwd = os.path.join(root, "forward")
    write_model(os.path.join(fwd, "model_true"), nx, nz, h, h, true)
    write_model(os.path.join(fwd, "model_init"), nx, nz, h, h, init)
    np.savetxt(os.path.join(fwd, "sources.dat"),
               [[(s + 0.5) * nx / shots * h, 10 * h, 0, 8.0, 0.15, 0.0, 1e10] for s in range(shots)])
    np.savetxt(os.path.join(fwd, "stations.dat"), [[(r + 0.5) * nx / nrec * h, 12 * h] for r in range(nrec)])
    with open(os.path.join(fwd, "config.ini"), "w") as f:
        f.write("[workflow]\nmode = forward\nmpi = no\n\n[solver]\nmethod = b200\nsh = no\npsv = yes\n"
                "nt = %d\ndt = %g\nabs_top = no\nabs_bottom = yes\nabs_left = yes\nabs_right = yes\n"
                "abs_width = 20\nabs_alpha = 0.015\nsave_coordinates =\nsave_snapshot = 0\n"
                "threads_per_block = 256\ncombine_sources = yes\n\n[path]\noutput = output\n"
                "model_init = model_init\nmodel_true = model_true\nsources = sources.dat\n"
                "stations = stations.dat\n" % (nt, dt))
    os.makedirs(os.path.join(root, "adjoint"), exist_ok=True)
    with open(os.path.join(root, "adjoint", "config.ini"), "w") as f:
        f.write("[workflow]\nmode = adjoint\ninherit = forward\nmpi = no\n\n[solver]\ncombine_sources = no\n"
                "adjoint_interval = %d\nsmooth = %d\n\n[postprocess]\nmethod = default\n\n[path]\noutput = output\n"
                % (sae, sigma))
    os.makedirs(os.path.join(root, "inverse"), exist_ok=True)
    with open(os.path.join(root, "inverse", "config.ini"), "w") as f:
        f.write("[workflow]\nmode = inversion\ninherit = adjoint\n\n[solver]\ninvert = %s\n\n[optimize]\nniter = %d\n"
                "method = %s\nls_step = 10\nls_step_max = 0.5\nls_step_init = 0.05\nls_thresh = 1.2\nlbfgs_mem = 5\n"
                "%s\n[path]\noutput = output\n" % (invert, niter, method, optimize_extra))
    return true["vp"], true["vs"], 2600.0 * true["vs"] ** 2


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--nz", type=int, default=512)
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--nrec", type=int, default=256)
    ap.add_argument("--nt", type=int, default=6000)
    ap.add_argument("--niter", type=int, default=20)
    ap.add_argument("--sigma", type=int, default=4)
    ap.add_argument("--sae", type=int, default=10)
    ap.add_argument("--invert", default="vp_vs", choices=["mu", "vp_vs"],
                    help="model variables: vp_vs (both perturbed velocities) or mu (the reference's)")
    a = ap.parse_args(argv)
    from . import workflow
    root = tempfile.mkdtemp()
    vp_true, vs_true, mu_true = write_case(root, a.nx, a.nz, a.shots, a.nrec, a.nt, a.niter, a.sigma, a.sae,
                                           invert=a.invert)
    t0 = time.time()
    with contextlib.redirect_stdout(io.StringIO()):
        wf = workflow.main(["--workdir", os.path.join(root, "inverse")])
    total = time.time() - t0
    opt = wf.optimize
    hist = opt.history
    mis = [h["misfit"] for h in hist]
    t = [h["t"] for h in hist]
    t90 = next((t[k] for k in range(len(mis)) if mis[k] <= 0.1 * mis[0]), None)
    mu = wf.solver.mu.copy_to_host()
    vp, vs = (x[:, : a.nz].reshape(-1).cpu().numpy() for x in wf.solver._velocities())

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    line = {"workload": "psv_inversion_%dx%d_shots%d_nt%d_lbfgs%d" % (a.nx, a.nz, a.shots, a.nt, a.niter),
            "invert": a.invert, "cells_per_gradient": 2 * a.shots * a.nx * a.nz * a.nt, "total_s": total,
            "s_per_iteration": (t[-1] - t[0]) / max(1, len(t) - 1), "misfit": mis, "t": t,
            "misfit_ratio_final": mis[-1] / mis[0], "time_to_90pct_drop_s": t90,
            "final_rel_err_vs_true": {"mu": rel(mu, mu_true), "vp": rel(vp, vp_true), "vs": rel(vs, vs_true)}}
    print(json.dumps(line))
    return line


if __name__ == "__main__":
    main()
