"""Exact discrete adjoint (fwi_run_transposed) and the autograd.Function.

The reference derivative is a central finite difference of the FP64
oracle's misfit chi = sum taper^2 (s - d)^2, so it carries no float32 noise;
the GPU gradient is the exact transpose of the float32 forward with FP64
accumulation.  Checked per cell at 16 random interior cells and along a
random smooth direction, for lambda, mu and rho, SH and P-SV, with
checkpointing segments shorter than nt.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle.oracle import Oracle, source_time_functions  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _case(mode, seed=3, nx=40, nz=36, nt=260):
    from seispie_b200.adjoint import AcquisitionSetup
    from seispie_b200.engine import Grid
    rng = np.random.default_rng(seed)
    h, dt = 10.0, 1e-3
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    smooth = lambda a, b, c: np.sin(a * i / nx + b * j / nz + c)  # noqa: E731
    vp = (3000 + 150 * smooth(3.1, 2.2, 0.3)).astype(np.float32)
    vs = (1732 + 120 * smooth(2.3, 3.7, 1.1)).astype(np.float32)
    rho = (2600 + 100 * smooth(1.7, 2.9, 2.0)).astype(np.float32)
    src = np.array([[120.0, 150.0, 0, 14.0, 0.07, 25.0, 1e10], [260.0, 90.0, 0, 12.0, 0.08, -40.0, 1e10]])
    rec = np.array([[50.0 + 45 * r, 30.0 + 40 * (r % 3)] for r in range(6)])
    absorb = (8, 0.05, 1, 1, 1, 0)
    setup = AcquisitionSetup(mode, Grid(nx, nz, h, h), dt, nt, src, rec, absorb, segment=37)
    lam = rho * (vp * vp - 2 * vs * vs)
    mu = rho * vs * vs
    return setup, dict(lam=lam, mu=mu, rho=rho), src, rec, absorb, rng


def _oracle_chi(setup, p, src, absorb, data):
    """chi of the FP64 oracle for params p (numpy [nx, nz])."""
    from seispie_b200.adjoint import hann_taper
    o = Oracle("f64")
    g = setup.grid
    params = dict(rho=p["rho"].ravel(), lam=p["lam"].ravel(), mu=p["mu"].ravel(),
                  bound=o.set_bound(g.nx, g.nz, *absorb))
    stf = source_time_functions(src, setup.nt, setup.dt)
    w = hann_taper(setup.nt, setup.dt) ** 2
    comps = "y" if setup.mode == 0 else "xz"
    chi = 0.0
    for s in range(setup.nshots):
        obs, _, _ = o.forward("sh" if setup.mode == 0 else "psv", g.nx, g.nz, g.dx, g.dz, setup.dt, setup.nt, params,
                              setup.src_id, stf, s, setup.rec_id)
        for ci, c in enumerate(comps):
            r = obs[c].reshape(-1, setup.nt) - data[ci, s]
            chi += float((w * r * r).sum())
    return chi


def _gpu_grad(setup, p, data):
    from seispie_b200.adjoint import Seismograms, waveform_misfit
    t = {k: torch.tensor(v, device="cuda", requires_grad=True) for k, v in p.items()}
    tr = Seismograms.apply(t["lam"], t["mu"], t["rho"], setup)
    chi = waveform_misfit(tr, torch.as_tensor(data, device="cuda"), setup.dt)
    chi.backward()
    return {k: v.grad.double().cpu().numpy() for k, v in t.items()}, chi.item()


def _data(setup, p, src, absorb):
    """Observed data: FP64 oracle traces of a perturbed model, [ncomp, nshots, nrec, nt]."""
    o = Oracle("f64")
    g = setup.grid
    q = {k: v.copy() for k, v in p.items()}
    q["mu"] = q["mu"] * (1 + 0.03 * np.cos(np.arange(q["mu"].size).reshape(q["mu"].shape) * 0.37))
    params = dict(rho=q["rho"].ravel(), lam=q["lam"].ravel(), mu=q["mu"].ravel(),
                  bound=o.set_bound(g.nx, g.nz, *absorb))
    stf = source_time_functions(src, setup.nt, setup.dt)
    comps = "y" if setup.mode == 0 else "xz"
    out = np.zeros((len(comps), setup.nshots, len(setup.rec_id), setup.nt))
    for s in range(setup.nshots):
        obs, _, _ = o.forward("sh" if setup.mode == 0 else "psv", g.nx, g.nz, g.dx, g.dz, setup.dt, setup.nt, params,
                              setup.src_id, stf, s, setup.rec_id)
        for ci, c in enumerate(comps):
            out[ci, s] = obs[c].reshape(-1, setup.nt)
    return out


@pytest.mark.parametrize("mode", ["sh", "psv"])
def test_exact_gradient_matches_fp64_finite_differences_per_cell(mode):
    setup, p, src, rec, absorb, rng = _case(mode)
    data = _data(setup, p, src, absorb)
    grad, _ = _gpu_grad(setup, p, data)
    g = setup.grid
    cells = [(int(rng.integers(4, g.nx - 4)), int(rng.integers(4, g.nz - 4))) for _ in range(16)]
    names = ["mu", "rho"] + (["lam"] if mode == "psv" else [])
    for name in names:
        scale = np.abs(grad[name]).max()
        for (ci, cj) in cells:
            h = 1e-4 * float(p[name][ci, cj])
            pp = {k: v.astype(np.float64).copy() for k, v in p.items()}
            pm = {k: v.astype(np.float64).copy() for k, v in p.items()}
            pp[name][ci, cj] += h
            pm[name][ci, cj] -= h
            fd = (_oracle_chi(setup, pp, src, absorb, data) - _oracle_chi(setup, pm, src, absorb, data)) / (2 * h)
            got = grad[name][ci, cj]
            assert abs(got - fd) <= 1e-3 * scale + 1e-3 * abs(fd), (name, ci, cj, got, fd, scale)


@pytest.mark.parametrize("mode", ["sh", "psv"])
def test_exact_gradient_directional_derivative(mode):
    setup, p, src, rec, absorb, rng = _case(mode, seed=5)
    data = _data(setup, p, src, absorb)
    grad, _ = _gpu_grad(setup, p, data)
    g = setup.grid
    i, j = np.meshgrid(np.arange(g.nx), np.arange(g.nz), indexing="ij")
    direction = {k: (0.5 + 0.5 * np.sin(0.21 * i + 0.13 * j + n)) * p[k] for n, k in enumerate(p)}
    eps = 1e-5
    pp = {k: p[k].astype(np.float64) + eps * direction[k] for k in p}
    pm = {k: p[k].astype(np.float64) - eps * direction[k] for k in p}
    fd = (_oracle_chi(setup, pp, src, absorb, data) - _oracle_chi(setup, pm, src, absorb, data)) / (2 * eps)
    dd = sum(float((grad[k] * direction[k]).sum()) for k in p)
    assert abs(dd - fd) < 1e-4 * abs(fd), (dd, fd)


def test_autograd_through_vp_vs_rho():
    """Gradients w.r.t. (vp, vs, rho) through the differentiable vps2lm."""
    from seispie_b200.adjoint import Seismograms, vps_to_lame, waveform_misfit
    setup, p, src, rec, absorb, rng = _case("psv", seed=9, nt=200)
    data = _data(setup, p, src, absorb)
    rho = p["rho"]
    vs = np.sqrt(p["mu"] / rho)
    vp = np.sqrt((p["lam"] + 2 * p["mu"]) / rho)
    t = {k: torch.tensor(v.astype(np.float32), device="cuda", requires_grad=True)
         for k, v in dict(vp=vp, vs=vs, rho=rho).items()}
    lam, mu = vps_to_lame(t["vp"], t["vs"], t["rho"])
    chi = waveform_misfit(Seismograms.apply(lam, mu, t["rho"], setup), torch.as_tensor(data, device="cuda"), setup.dt)
    chi.backward()
    gvs = t["vs"].grad.double().cpu().numpy()
    # directional check in vs
    d = np.ones_like(vs) * 5.0
    eps = 1e-3

    def chi_of(vsn):
        vsn = vsn.astype(np.float64)
        rr, vpp = rho.astype(np.float64), vp.astype(np.float64)
        q = dict(rho=rr, lam=rr * (vpp * vpp - 2 * vsn * vsn), mu=rr * vsn * vsn)
        return _oracle_chi(setup, q, src, absorb, data)

    fd = (chi_of(vs + eps * d) - chi_of(vs - eps * d)) / (2 * eps)
    assert abs(float((gvs * d).sum()) - fd) < 1e-3 * abs(fd)
