"""GPU optimizers (seispie_b200.optimize) against the reference's own
L-BFGS / CG trajectories (tests/golden/optimize.npz, made by running
seispie/optimize/*.py), the FP64 vector kernels, and a small inversion
through the sprun-compatible runner with the b200 solver."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from tests.conftest import load_golden  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_vector_kernels_fp64():
    from seispie_b200.optimize.vec import VecOps
    rng = np.random.default_rng(0)
    ops = VecOps(torch.device("cuda"))
    for n in (1, 1000, 262144 + 17):
        x = rng.standard_normal(n).astype(np.float32)
        y = rng.standard_normal(n).astype(np.float32)
        tx, ty = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
        ref = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
        assert abs(ops.dot(tx, ty) - ref) <= 1e-12 * max(1.0, np.abs(x).dot(np.abs(y)))
        assert ops.absmax(tx) == float(np.abs(x).max())
        out = ops.axpby(0.3, tx, -1.7, ty).cpu().numpy()
        assert np.array_equal(out, (0.3 * x.astype(np.float64) - 1.7 * y.astype(np.float64)).astype(np.float32))
    assert ops.dot(tx, ty) == ops.dot(tx, ty)  # deterministic


class DeviceStandIn:
    """Quadratic misfit with the b200 solver's device-side API."""

    def __init__(self, w, mt, m0):
        self.w, self.mt = w, mt
        self.m = torch.as_tensor(m0).cuda()
        self.device = self.m.device
        self.trials = 0

    def update_model_device(self, m):
        self.m = m.clone()
        self.trials += 1

    def compute_misfit(self):
        m = self.m.double().cpu().numpy()
        return float(np.sum(self.w * (m - self.mt) ** 2))

    def gradient(self):
        m = self.m.double().cpu().numpy()
        return torch.as_tensor((2 * self.w * (m - self.mt)).astype(np.float32)).cuda()


@pytest.mark.parametrize("name", ["lbfgs", "cg"])
def test_optimizer_follows_reference_trajectory(name):
    from seispie_b200 import optimize
    g = load_golden("optimize")
    s = DeviceStandIn(g["w"], g["mt"], g["m0"])

    class Workflow:
        pass

    wf = Workflow()
    wf.solver = s
    opt = getattr(optimize, name)()
    opt.config = dict(niter="6", ls_step="10", ls_step_max="0.5", ls_step_init="0.05", ls_thresh="1.2",
                      lbfgs_mem="3")
    opt.mpi = None
    opt.setup(wf)
    # The reference takes its dot products in float32 (np.dot of float32
    # arrays), these are FP64: decisions must agree exactly, vectors to the
    # float32-dot error (directions 2e-4 of their max-norm, models 1e-6).
    for i in range(len(g[name + "_status"])):
        opt.g_new, misfit, opt.m_new = s.gradient(), s.compute_misfit(), s.m.clone()
        np.testing.assert_allclose(misfit, g[name + "_misfit"][i], rtol=1e-4)
        opt.p_new = opt.compute_direction()
        pr = g[name + "_p"][i]
        np.testing.assert_allclose(opt.p_new.cpu().numpy(), pr, rtol=0, atol=2e-4 * np.abs(pr).max())
        opt.m_old, opt.p_old, opt.g_old = opt.m_new, opt.p_new, opt.g_new
        status = opt.line_search(misfit)
        assert status == g[name + "_status"][i]
        assert s.trials == g[name + "_ntrials"][i]
        mr = g[name + "_m"][i]
        np.testing.assert_allclose(s.m.cpu().numpy(), mr, rtol=0, atol=1e-6 * np.abs(mr).max())


def _write_inversion_case(root):
    """A small SH checkerboard inversion laid out like the reference's
    examples (forward <- adjoint <- inverse, with config inheritance)."""
    from seispie_b200.io import write_model
    nx, nz, h = 48, 40, 10.0
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    vs_true = 1732 * (1 + 0.06 * np.sign(np.sin(np.pi * i / 12) * np.sin(np.pi * j / 12) + 1e-9))
    for d, vs in (("model_true", vs_true.ravel()), ("model_init", np.full(nx * nz, 1732.0))):
        write_model(os.path.join(root, "forward", d), nx, nz, h, h,
                    dict(vp=np.full(nx * nz, 3000.0), vs=vs, rho=np.full(nx * nz, 2600.0)))
    np.savetxt(os.path.join(root, "forward", "sources.dat"),
               [[x, 30.0, 0, 15.0, 0.07, 0.0, 1e10] for x in (60.0, 160.0, 260.0, 360.0)])
    np.savetxt(os.path.join(root, "forward", "stations.dat"), [[x, 360.0] for x in np.arange(20.0, 460.0, 20.0)])
    open(os.path.join(root, "forward", "config.ini"), "w").write(
        "[workflow]\nmode = forward\nmpi = no\n\n[solver]\nmethod = b200\nsh = yes\npsv = no\nnt = 500\n"
        "dt = 0.001\nabs_top = no\nabs_bottom = yes\nabs_left = yes\nabs_right = yes\nabs_width = 10\n"
        "abs_alpha = 0.04\nsave_coordinates =\nsave_snapshot = 0\nthreads_per_block = 256\ncombine_sources = yes\n\n"
        "[path]\noutput = output\nmodel_init = model_init\nmodel_true = model_true\nsources = sources.dat\n"
        "stations = stations.dat\n")
    os.makedirs(os.path.join(root, "adjoint"))
    open(os.path.join(root, "adjoint", "config.ini"), "w").write(
        "[workflow]\nmode = adjoint\ninherit = forward\nmpi = no\n\n[solver]\ncombine_sources = no\n"
        "adjoint_interval = 5\nsmooth = 2\n\n[postprocess]\nmethod = default\n\n[path]\noutput = output\n")
    os.makedirs(os.path.join(root, "inverse"))
    open(os.path.join(root, "inverse", "config.ini"), "w").write(
        "[workflow]\nmode = inversion\ninherit = adjoint\n\n[optimize]\nniter = 3\nmethod = lbfgs\nls_step = 10\n"
        "ls_step_max = 0.5\nls_step_init = 0.05\nls_thresh = 1.2\nlbfgs_mem = 5\n\n[path]\noutput = output\n")


def test_inversion_through_runner_reduces_misfit(tmp_path):
    from seispie_b200 import workflow
    _write_inversion_case(str(tmp_path))
    wf = workflow.main(["--workdir", os.path.join(str(tmp_path), "inverse")])
    mis = wf.optimize.misfits
    assert mis[0] == 1.0 and mis[-1] < 0.7, mis
    out = os.path.join(str(tmp_path), "inverse", "output")
    assert os.path.exists(os.path.join(out, "proc000003_mu.bin"))


def test_joint_vp_vs_inversion_through_runner(tmp_path):
    """invert = vp_vs: a P-SV case with both vp and vs perturbed; L-BFGS on
    [vp; vs] (gradients from the exact kernels by the chain rule) lowers the
    misfit and moves both velocities towards the true model."""
    from seispie_b200 import workflow
    from seispie_b200.io import write_model
    root = str(tmp_path)
    nx, nz, h = 48, 40, 10.0
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    board = np.sign(np.sin(np.pi * i / 12) * np.sin(np.pi * j / 12) + 1e-9).ravel()
    vp_true, vs_true = 3000 * (1 + 0.05 * board), 1732 * (1 - 0.05 * board)
    n = nx * nz
    write_model(os.path.join(root, "forward", "model_true"), nx, nz, h, h,
                dict(vp=vp_true, vs=vs_true, rho=np.full(n, 2600.0)))
    write_model(os.path.join(root, "forward", "model_init"), nx, nz, h, h,
                dict(vp=np.full(n, 3000.0), vs=np.full(n, 1732.0), rho=np.full(n, 2600.0)))
    np.savetxt(os.path.join(root, "forward", "sources.dat"),
               [[x, 30.0, 0, 15.0, 0.07, 20.0, 1e10] for x in (60.0, 160.0, 260.0, 360.0)])
    np.savetxt(os.path.join(root, "forward", "stations.dat"), [[x, 360.0] for x in np.arange(20.0, 460.0, 20.0)])
    open(os.path.join(root, "forward", "config.ini"), "w").write(
        "[workflow]\nmode = forward\nmpi = no\n\n[solver]\nmethod = b200\nsh = no\npsv = yes\nnt = 500\n"
        "dt = 0.001\nabs_top = no\nabs_bottom = yes\nabs_left = yes\nabs_right = yes\nabs_width = 10\n"
        "abs_alpha = 0.04\nsave_coordinates =\nsave_snapshot = 0\nthreads_per_block = 256\ncombine_sources = yes\n\n"
        "[path]\noutput = output\nmodel_init = model_init\nmodel_true = model_true\nsources = sources.dat\n"
        "stations = stations.dat\n")
    os.makedirs(os.path.join(root, "adjoint"))
    open(os.path.join(root, "adjoint", "config.ini"), "w").write(
        "[workflow]\nmode = adjoint\ninherit = forward\nmpi = no\n\n[solver]\ncombine_sources = no\n"
        "adjoint_interval = 5\nsmooth = 2\n\n[postprocess]\nmethod = default\n\n[path]\noutput = output\n")
    os.makedirs(os.path.join(root, "inverse"))
    open(os.path.join(root, "inverse", "config.ini"), "w").write(
        "[workflow]\nmode = inversion\ninherit = adjoint\n\n[solver]\ninvert = vp_vs\n\n[optimize]\nniter = 4\n"
        "method = lbfgs\nls_step = 10\nls_step_max = 0.5\nls_step_init = 0.05\nls_thresh = 1.2\nlbfgs_mem = 5\n\n"
        "[path]\noutput = output\n")
    wf = workflow.main(["--workdir", os.path.join(root, "inverse")])
    mis = wf.optimize.misfits
    assert mis[-1] < 0.8 * mis[0], mis
    m = wf.solver.model_vector_device().cpu().numpy()
    for got, true, start in ((m[:n], vp_true, 3000.0), (m[n:], vs_true, 1732.0)):
        assert np.linalg.norm(got - true) < np.linalg.norm(start - true)
    out = os.path.join(root, "inverse", "output")
    assert os.path.exists(os.path.join(out, "proc000004_vp.bin")) and os.path.exists(os.path.join(out, "proc000004_vs.bin"))
