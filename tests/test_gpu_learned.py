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
