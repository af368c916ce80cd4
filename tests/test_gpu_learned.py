"""The learned-preconditioner optimizer (``method = lbfgs_learned``) on a
small P-SV inversion: recorded training pairs are consistent with the
inversion history, and with a network that has not been trained the
optimizer still descends (each learned direction is either accepted by the
line search or replaced by the L-BFGS direction)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


NX, NZ, SHOTS, NT, NITER = 128, 64, 8, 800, 3


def test_recorded_pairs_and_untrained_network_fallback(tmp_path):
    from seispie_b200.learned import features, random_board, run_inversion
    from seispie_b200.unet import UNet
    board = random_board(np.random.default_rng(3), NX, NZ)
    rec = str(tmp_path / "pairs.npz")
    opt, _, mu_true = run_inversion(str(tmp_path / "a"), NX, NZ, SHOTS, NT, NITER, board, 0.06, "lbfgs_learned",
                                    "record_pairs = %s\n" % rec)
    assert mu_true.size == NX * NZ
    z = np.load(rec)
    n = len(z["g"])
    assert n == NITER and int(z["nx"]) == NX and int(z["nz"]) == NZ
    for key in ("g", "illum", "m", "d"):
        assert z[key].shape == (n, NX * NZ) and np.isfinite(z[key]).all()
    assert (z["illum"] >= 0).all() and z["illum"].max() > 0
    # the accepted update of iteration k takes the model of k to the model of k+1
    np.testing.assert_allclose(z["m"][0] + z["d"][0], z["m"][1], rtol=0, atol=1e-3 * np.abs(z["m"][1]).max())
    mis = [h["misfit"] for h in opt.history if "misfit" in h]
    assert mis[-1] < mis[0]
    # features of a recorded iteration: normalised channels, zero padding
    f = features(*(torch.as_tensor(z[k][1], device="cuda") for k in ("g", "illum", "m")), NX, NZ)
    assert f.shape == (1, 3, NX, NZ) and float(f[0, 0].abs().max()) == pytest.approx(1.0)
    assert 0.0 <= float(f[0, 1].min()) and float(f[0, 1].max()) == pytest.approx(1.0, abs=1e-4)
    # an untrained network: the optimizer falls back where needed and still descends
    w = str(tmp_path / "w.npz")
    UNet("cuda", seed=5).save(w)
    opt2, _, _ = run_inversion(str(tmp_path / "b"), NX, NZ, SHOTS, NT, NITER, board, 0.06, "lbfgs_learned",
                               "unet_weights = %s\n" % w)
    mis2 = [h["misfit"] for h in opt2.history if "misfit" in h]
    assert opt2.learned_accepted + opt2.learned_rejected >= NITER - 1
    assert all(b <= a * (1 + 1e-9) for a, b in zip(mis2, mis2[1:]))
    assert mis2[-1] < mis2[0]
    assert os.path.exists(w)


def _count_solves(monkeypatch):
    """Record every misfit evaluation (one forward solve) and gradient
    (forward + adjoint: two solves) of the b200 solver, with its misfit."""
    from seispie_b200.solver import b200 as Solver
    log = []
    misfit, gradient = Solver.compute_misfit, Solver.compute_gradient_device

    def counted_misfit(self):
        r = misfit(self)
        log.append((1, float(r)))
        return r

    def counted_gradient(self):
        r = gradient(self)
        log.append((2, float(r[1])))
        return r

    monkeypatch.setattr(Solver, "compute_misfit", counted_misfit)
    monkeypatch.setattr(Solver, "compute_gradient_device", counted_gradient)
    return log


def _solves_to_drop(log, frac):
    cost = 0
    for n, m in log:
        cost += n
        if m <= (1 - frac) * log[0][1]:
            return cost
    return None


def test_trained_weights_reach_90pct_drop_with_fewer_solves(tmp_path, monkeypatch):
    """What the shipped model-error weights (unet_psv_mu_error.npz, with the
    number of learned iterations stored beside them) gain over plain L-BFGS
    on a fixed held-out case of their training geometry: a random model
    (seed 4242), 256 x 128 cells, 16 shots, nt 1500, only mu perturbed (8 %),
    20 iterations.  Counted in wave solves (a misfit evaluation is one, a
    gradient two), the learned run reaches a 90 % misfit drop in at most
    0.75 of the solves plain L-BFGS needs (31 against 53 on a B200), and
    ends with a smaller model error to the true mu."""
    from seispie_b200.io import read_field
    from seispie_b200.learned import ERROR_WEIGHTS, random_board, run_inversion
    nx, nz, shots, nt, niter = 256, 128, 16, 1500, 20
    board = random_board(np.random.default_rng(4242), nx, nz)
    log = _count_solves(monkeypatch)
    res = {}
    for label, method, extra in (("plain", "lbfgs", ""),
                                 ("learned", "lbfgs_learned", "unet_weights = %s\n" % ERROR_WEIGHTS)):
        log.clear()
        root = str(tmp_path / label)
        opt, _, mu_true = run_inversion(root, nx, nz, shots, nt, niter, board, 0.08, method, extra, perturb="mu")
        _, mu = read_field(os.path.join(root, "inverse", "output", "proc%06d_mu.bin" % niter))
        mt = np.asarray(mu_true, np.float64).ravel()
        res[label] = dict(solves=_solves_to_drop(log, 0.9), final=log[-1][1] / log[0][1],
                          err=float(np.linalg.norm(mu - mt) / np.linalg.norm(mt)),
                          accepted=getattr(opt, "learned_accepted", 0))
    plain, learned = res["plain"], res["learned"]
    assert plain["solves"] is not None and learned["solves"] is not None, res
    assert learned["accepted"] >= 1, res
    assert learned["solves"] <= 0.75 * plain["solves"], res
    assert learned["final"] < plain["final"] and learned["err"] < plain["err"], res


def test_weights_trained_at_512x256_gain_there(tmp_path, monkeypatch):
    """The model-error weights trained in the 512 x 256, 32-shot geometry
    (unet_psv_mu_error_512.npz) on a held-out random model of that geometry
    (seed 31337, nt 2500, mu-only 8 %, 20 iterations): the learned run
    reaches a 50 % misfit drop in at most half the wave solves plain L-BFGS
    needs (or plain does not reach it at all) and ends at a misfit well below
    plain L-BFGS's (0.20 against 0.49 on a B200)."""
    from seispie_b200.learned import ERROR_WEIGHTS_512, random_board, run_inversion
    nx, nz, shots, nt, niter = 512, 256, 32, 2500, 20
    board = random_board(np.random.default_rng(31337), nx, nz)
    log = _count_solves(monkeypatch)
    res = {}
    for label, method, extra in (("plain", "lbfgs", ""),
                                 ("learned", "lbfgs_learned", "unet_weights = %s\n" % ERROR_WEIGHTS_512)):
        log.clear()
        opt, _, _ = run_inversion(str(tmp_path / label), nx, nz, shots, nt, niter, board, 0.08, method, extra,
                                  perturb="mu")
        res[label] = dict(solves=_solves_to_drop(log, 0.5), final=log[-1][1] / log[0][1],
                          accepted=getattr(opt, "learned_accepted", 0))
    plain, learned = res["plain"], res["learned"]
    assert learned["accepted"] >= 1 and learned["solves"] is not None, res
    assert plain["solves"] is None or learned["solves"] <= 0.5 * plain["solves"], res
    assert learned["final"] < 0.6 * plain["final"], res
