"""Learned preconditioner for the inversion: data, training and evaluation.

    python -m seispie_b200.learned gen   --out DIR [--cases 60 --nx 256 --nz 128 --shots 16 --nt 1500 --niter 10]
    python -m seispie_b200.learned train --data DIR --weights W.npz [--epochs 30]
    python -m seispie_b200.learned eval  [--weights W.npz --nx 512 --nz 256 --shots 32 --nt 2500 --niter 12]

gen runs plain L-BFGS inversions (the reference's step logic, exact P-SV
gradient, mu as the model variable as in the reference's workflow) on random
checkerboard and smooth-layer models and records, per iteration, the
smoothed gradient, the source illumination, the model and the accepted
update m_{k+1} - m_k (and the case's true mu).  train fits the BF16 U-Net
(seispie_b200.unet) to map the first three to the direction of the fourth
(each normalised, MSE loss, Adam); ``--target error`` trains on the model
error m_true - m_k instead.  eval runs the same inversion twice, plain and with
``method = lbfgs_learned`` (the learned direction where it is a descent
direction and passes the line search, L-BFGS otherwise), and prints both
misfit histories with wall-clock times, the time to a 50 % and a 90 % misfit
drop, and how often the learned direction was used.
"""
from __future__ import annotations

import argparse
import contextlib
import glob
import io
import json
import math
import os
import tempfile
import time

import numpy as np
import torch

from .unet import UNet


# weights trained by ``gen`` + ``train`` (about 1500 pairs of 256 x 128 P-SV mu
# inversions, 30 epochs): on the accepted L-BFGS updates (the default), and on
# the model error of mu-only cases (``--perturb mu``, ``--target error``)
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_psv_mu.npz")
ERROR_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_psv_mu_error.npz")
# the model-error target trained on about 860 pairs of 512 x 256, 32-shot, nt 2500 mu inversions
ERROR_WEIGHTS_512 = os.path.join(WEIGHTS_DIR, "unet_psv_mu_error_512.npz")


def _pad8(n: int) -> int:
    return (n + 7) // 8 * 8


def features(g: torch.Tensor, illum: torch.Tensor, m: torch.Tensor, nx: int, nz: int) -> torch.Tensor:
    """Network input [1, 3, H, W] (H, W = nx, nz rounded up to 8, zero
    padding): gradient / max|gradient|, log10 of the relative illumination
    mapped to [0, 1] (1e-4 of the peak -> 0), model / mean(model) - 1."""
    dev = g.device
    out = torch.zeros((1, 3, _pad8(nx), _pad8(nz)), dtype=torch.float32, device=dev)
    gg, ii, mm = (t.reshape(nx, nz).float() for t in (g, illum, m))
    out[0, 0, :nx, :nz] = gg / gg.abs().max().clamp_min(1e-30)
    out[0, 1, :nx, :nz] = torch.log10(ii / ii.max().clamp_min(1e-30) + 1e-4) / 4.0 + 1.0
    out[0, 2, :nx, :nz] = mm / mm.mean().clamp_min(1e-30) - 1.0
    return out


class Preconditioner:
    """A trained U-Net applied to one iteration's (gradient, illumination, model)."""

    def __init__(self, net: UNet):
        self.net = net
        # number of iterations the network's direction is meant for (None: the optimizer's default)
        self.learned_iterations = getattr(net, "meta", {}).get("learned_iterations")

    @classmethod
    def load(cls, path: str, device="cuda") -> "Preconditioner":
        return cls(UNet.load(path, device))

    def direction(self, g, illum, m, nx: int, nz: int, scale: float) -> torch.Tensor:
        """Update direction (float32 vector of nx*nz) with max-norm `scale`."""
        out = self.net.forward(features(g, illum, m, nx, nz))[0, :nx, :nz]
        peak = float(out.abs().max())
        if not peak > 0:
            return torch.zeros(nx * nz, dtype=torch.float32, device=g.device)
        return (out * (scale / peak)).reshape(-1).contiguous()


# ------------------------------------------------------------------ cases

def random_board(rng, nx: int, nz: int) -> np.ndarray:
    """A perturbation pattern in [-1, 1]: a checkerboard with random square
    size and offset, or smooth dipping layers."""
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    if rng.random() < 0.6:
        sq = int(rng.choice([16, 24, 32, 48, 64]))
        oi, oj = rng.integers(0, sq, 2)
        return np.where((((i + oi) // sq) + ((j + oj) // sq)) % 2 == 0, 1.0, -1.0)
    lam = rng.uniform(20, 60)
    dip = rng.uniform(-0.3, 0.3)
    return np.sin(2 * np.pi * (j + dip * i) / lam + rng.uniform(0, 2 * np.pi))


def run_inversion(root: str, nx: int, nz: int, shots: int, nt: int, niter: int, board, amp: float, method: str,
                  extra: str = "", sigma: int = 4, nrec: int | None = None, perturb: str = "both"):
    """One inversion through the workflow; returns (optimizer, wall seconds,
    true mu of the case)."""
    from . import workflow
    from .inversion_bench import write_case
    _, _, mu_true = write_case(root, nx, nz, shots, nrec or max(16, nx // 4), nt, niter, sigma, 10, board=board,
                               amp=amp, method=method, optimize_extra=extra, perturb=perturb)
    t0 = time.time()
    with contextlib.redirect_stdout(io.StringIO()):
        wf = workflow.main(["--workdir", os.path.join(root, "inverse")])
    return wf.optimize, time.time() - t0, mu_true


def cmd_gen(a):
    os.makedirs(a.out, exist_ok=True)
    rng = np.random.default_rng(a.seed)
    t0 = time.time()
    npairs = 0
    for c in range(a.cases):
        board = random_board(rng, a.nx, a.nz)
        amp = float(rng.uniform(0.03, 0.08))
        path = os.path.abspath(os.path.join(a.out, "pairs_%04d.npz" % c))
        with tempfile.TemporaryDirectory() as root:
            try:
                _, _, mu_true = run_inversion(root, a.nx, a.nz, a.shots, a.nt, a.niter, board, amp,
                                              "lbfgs_learned", "record_pairs = %s\n" % path, perturb=a.perturb)
            except RuntimeError as e:  # the reference's line search gives up on a non-convex fit: skip the case
                print(json.dumps({"case": c, "skipped": str(e)}), flush=True)
                continue
        if os.path.exists(path):
            z = dict(np.load(path))
            z["m_true"] = np.asarray(mu_true, np.float32).ravel()  # for the model-error target
            np.savez(path, **z)
            npairs += len(z["g"])
        print(json.dumps({"case": c, "pairs": npairs, "seconds": time.time() - t0}), flush=True)
        if a.max_seconds and time.time() - t0 > a.max_seconds:
            break
    print(json.dumps({"cases": c + 1, "pairs": npairs, "seconds": time.time() - t0}))


def load_pairs(data_dir: str, device, target: str = "update"):
    """Inputs and targets of every recorded iteration.  target "update": the
    accepted L-BFGS update m_{k+1} - m_k; "error": the model error
    m_true - m_k (synthetic cases only)."""
    X, Y = [], []
    for f in sorted(glob.glob(os.path.join(data_dir, "pairs_*.npz"))):
        z = np.load(f)
        nx, nz = int(z["nx"]), int(z["nz"])
        for k in range(len(z["g"])):
            g, i, m, d = (torch.as_tensor(z[key][k], device=device) for key in ("g", "illum", "m", "d"))
            if target == "error":
                d = torch.as_tensor(z["m_true"], device=device) - m
            if not float(d.abs().max()) > 0:
                continue
            X.append(features(g, i, m, nx, nz)[0])
            t = torch.zeros((_pad8(nx), _pad8(nz)), dtype=torch.float32, device=device)
            t[:nx, :nz] = (d / d.abs().max()).reshape(nx, nz)
            Y.append(t)
    return torch.stack(X), torch.stack(Y)


def _cosine(a, b):
    a, b = a.reshape(a.shape[0], -1), b.reshape(b.shape[0], -1)
    return (a * b).sum(1) / (a.norm(dim=1) * b.norm(dim=1)).clamp_min(1e-30)


def cmd_train(a):
    dev = torch.device("cuda")
    X, Y = load_pairs(a.data, dev, a.target)
    n = X.shape[0]
    gen = torch.Generator().manual_seed(a.seed)
    perm = torch.randperm(n, generator=gen).to(dev)
    nval = max(1, n // 10)
    val, tr = perm[:nval], perm[nval:]
    net = UNet(dev, seed=a.seed)
    t0 = time.time()
    steps = 0
    total = a.epochs * math.ceil(len(tr) / a.batch)
    log = []
    for ep in range(a.epochs):
        order = tr[torch.randperm(len(tr), generator=gen).to(dev)]
        run = 0.0
        for b0 in range(0, len(order), a.batch):
            idx = order[b0:b0 + a.batch]
            out = net.forward(X[idx])
            loss, gout = net.mse(out, Y[idx])
            net.backward(gout)
            lr = a.lr * 0.5 * (1 + math.cos(math.pi * steps / total))
            net.adam(lr)
            steps += 1
            run += float(loss) * len(idx)
        with torch.no_grad():
            pv = torch.cat([net.forward(X[val[k:k + a.batch]]) for k in range(0, nval, a.batch)])
            vloss = float(((pv - Y[val]) ** 2).mean())
            cos = _cosine(pv, Y[val])
            # descent rate: the prediction against the (normalised) gradient channel
            desc = float(((pv * X[val, 0]).reshape(nval, -1).sum(1) < 0).float().mean())
        log.append(dict(epoch=ep, train_loss=run / len(tr), val_loss=vloss, val_cosine=float(cos.mean()),
                        val_descent_rate=desc))
        print(json.dumps(log[-1]), flush=True)
    net.save(a.weights, target=a.target, learned_iterations=2 if a.target == "error" else 5)
    base = float((Y[val] ** 2).mean())
    print(json.dumps({"pairs": n, "target": a.target, "train": len(tr), "val": nval, "epochs": a.epochs,
                      "seconds": time.time() - t0,
                      "val_loss": log[-1]["val_loss"], "val_loss_zero_predictor": base,
                      "val_cosine": log[-1]["val_cosine"], "weights": a.weights}))


def _summary(opt, wall):
    hist = [h for h in opt.history if "misfit" in h]
    mis = [h["misfit"] for h in hist]
    t = [h["t"] for h in hist]

    def t_drop(frac):
        return next((t[k] for k in range(len(mis)) if mis[k] <= (1 - frac) * mis[0]), None)

    return dict(misfit=mis, t=t, wall_s=wall, final_ratio=mis[-1] / mis[0], time_to_50pct_drop_s=t_drop(0.5),
                time_to_90pct_drop_s=t_drop(0.9), learned_accepted=getattr(opt, "learned_accepted", 0),
                learned_rejected=getattr(opt, "learned_rejected", 0))


def cmd_eval(a):
    rng = np.random.default_rng(a.seed)
    board = random_board(rng, a.nx, a.nz) if a.random_model else None
    res = {}
    learned_extra = "unet_weights = %s\n" % os.path.abspath(a.weights)
    if a.learned_iterations:
        learned_extra += "learned_iterations = %d\n" % a.learned_iterations
    for label, method, extra in (("plain", "lbfgs", ""), ("learned", "lbfgs_learned", learned_extra)):
        with tempfile.TemporaryDirectory() as root:
            opt, wall, _ = run_inversion(root, a.nx, a.nz, a.shots, a.nt, a.niter, board, a.amp, method, extra,
                                         perturb=a.perturb)
        res[label] = _summary(opt, wall)
        print(json.dumps({label: res[label]}), flush=True)
    print(json.dumps({"workload": "psv_inversion_%dx%d_shots%d_nt%d_lbfgs%d_%s" % (a.nx, a.nz, a.shots, a.nt, a.niter,
                                                                                  a.perturb),
                      "plain_final_ratio": res["plain"]["final_ratio"],
                      "learned_final_ratio": res["learned"]["final_ratio"],
                      "plain_time_to_90pct_drop_s": res["plain"]["time_to_90pct_drop_s"],
                      "learned_time_to_90pct_drop_s": res["learned"]["time_to_90pct_drop_s"],
                      "plain_time_to_50pct_drop_s": res["plain"]["time_to_50pct_drop_s"],
                      "learned_time_to_50pct_drop_s": res["learned"]["time_to_50pct_drop_s"],
                      "learned_accepted": res["learned"]["learned_accepted"],
                      "learned_rejected": res["learned"]["learned_rejected"]}))


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gen")
    g.add_argument("--out", required=True)
    g.add_argument("--cases", type=int, default=60)
    g.add_argument("--nx", type=int, default=256)
    g.add_argument("--nz", type=int, default=128)
    g.add_argument("--shots", type=int, default=16)
    g.add_argument("--nt", type=int, default=1500)
    g.add_argument("--niter", type=int, default=10)
    g.add_argument("--seed", type=int, default=1)
    g.add_argument("--max-seconds", type=float, default=0, help="stop after this long (0: no limit)")
    g.add_argument("--perturb", default="both", choices=["both", "vs", "mu"])
    t = sub.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--weights", required=True)
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--batch", type=int, default=8)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--target", default="update", choices=["update", "error"],
                   help="update: the accepted L-BFGS update; error: the true model error of the synthetic case")
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--nx", type=int, default=512)
    e.add_argument("--nz", type=int, default=256)
    e.add_argument("--shots", type=int, default=32)
    e.add_argument("--nt", type=int, default=2500)
    e.add_argument("--niter", type=int, default=12)
    e.add_argument("--amp", type=float, default=0.08)
    e.add_argument("--random-model", action="store_true", help="random board instead of the 64-cell checkerboard")
    e.add_argument("--seed", type=int, default=12345)
    e.add_argument("--learned-iterations", type=int, default=0,
                   help="iterations that try the learned direction (0: the optimizer's default, lbfgs_mem)")
    e.add_argument("--perturb", default="both", choices=["both", "vs", "mu"],
                   help="mu: perturb only mu (lambda kept), so that the mu-only inversion can fit the data")
    a = ap.parse_args(argv)
    {"gen": cmd_gen, "train": cmd_train, "eval": cmd_eval}[a.cmd](a)


if __name__ == "__main__":
    main()
