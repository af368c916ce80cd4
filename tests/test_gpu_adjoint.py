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


def test_misfit_tracegrad_is_reversed_negated_adjoint_source():
    from seispie_b200 import engine
    rng = np.random.default_rng(4)
    ns, nrec, nt = 2, 5, 333
    d = torch.as_tensor(rng.standard_normal(ns * nrec * nt).astype(np.float32)).cuda()
    s = torch.as_tensor(rng.standard_normal(ns * nrec * nt).astype(np.float32)).cuda()
    ad, g = torch.empty_like(d), torch.empty_like(d)
    m1 = engine.misfit(d, s, ad, ns, nrec, nt, 2e-3)
    m2 = engine.misfit_tracegrad(d, s, g, ns, nrec, nt, 2e-3)
    assert torch.equal(m1, m2)
    assert torch.equal(g.view(ns, nrec, nt), -ad.view(ns, nrec, nt).flip(-1))


def test_plugin_psv_gradient_is_dt_times_exact(tmp_path):
    """compute_gradient of the b200 plugin for P-SV (exact adjoint by
    default) equals dt times the autograd gradient, before smoothing."""
    import os
    from seispie_b200.adjoint import AcquisitionSetup, Seismograms, waveform_misfit
    from seispie_b200.engine import Grid
    from seispie_b200.io import write_model
    from seispie_b200.solver import b200
    nx, nz, h, nt = 44, 38, 10.0, 240
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    vs_true = 1732 * (1 + 0.05 * np.sign(np.sin(i / 5.0) * np.sin(j / 5.0) + 1e-9))
    root = str(tmp_path)
    for d, vs in (("true", vs_true.ravel()), ("init", np.full(nx * nz, 1732.0))):
        write_model(os.path.join(root, d), nx, nz, h, h, dict(vp=np.full(nx * nz, 3000.0), vs=vs,
                                                              rho=np.full(nx * nz, 2600.0)))
    src = np.array([[100.0, 60.0, 0, 14.0, 0.07, 20.0, 1e10], [300.0, 60.0, 0, 14.0, 0.07, -30.0, 1e10]])
    rec = np.array([[30.0 + 30 * r, 80.0] for r in range(12)])
    np.savetxt(os.path.join(root, "src.dat"), src)
    np.savetxt(os.path.join(root, "rec.dat"), rec)
    os.makedirs(os.path.join(root, "out"))
    s = b200()
    s.config = dict(nt=str(nt), dt="1e-3", sh="no", psv="yes", abs_left="yes", abs_right="yes", abs_top="no",
                    abs_bottom="yes", abs_width="8", abs_alpha="0.05", save_coordinates="", combine_sources="no",
                    save_snapshot="0", adjoint_interval="4", smooth="2")
    s.path = dict(model_true=os.path.join(root, "true"), model_init=os.path.join(root, "init"),
                  sources=os.path.join(root, "src.dat"), stations=os.path.join(root, "rec.dat"),
                  output=os.path.join(root, "out"))
    s.mpi = None
    s.setup(None)
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.import_traces()
    s.import_model(0)
    s.compute_gradient()
    kraw = s.k_mu_f64[:, :nz].cpu().numpy()
    setup = AcquisitionSetup("psv", Grid(nx, nz, h, h), 1e-3, nt, src, rec, (8, 0.05, 1, 1, 1, 0))
    rho = torch.full((nx, nz), 2600.0, device="cuda")
    vp = torch.full((nx, nz), 3000.0, device="cuda")
    lam = rho * (vp * vp - 2 * 1732.0 ** 2)
    mu = (rho * 1732.0 ** 2).clone().requires_grad_(True)
    data = torch.stack([torch.as_tensor(np.stack(s.syn_x)).view(2, 12, nt),
                        torch.as_tensor(np.stack(s.syn_z)).view(2, 12, nt)]).cuda()
    chi = waveform_misfit(Seismograms.apply(lam, mu, rho, setup), data, setup.dt)
    chi.backward()
    ref = 1e-3 * mu.grad.double().cpu().numpy()
    assert np.linalg.norm(kraw - ref) / np.linalg.norm(ref) < 1e-5
    # a second call restages the observed traces into the same pinned buffers: same gradient
    s.compute_gradient()
    assert np.array_equal(s.k_mu_f64[:, :nz].cpu().numpy(), kraw)
    # one shot per batch: each batch restages into the buffers the previous one uploaded from
    s.batch_memory = 1.0
    s.compute_gradient()
    k1 = s.k_mu_f64[:, :nz].cpu().numpy()
    assert np.linalg.norm(k1 - kraw) / np.linalg.norm(kraw) < 1e-6


def test_trace_suffix_sum():
    from seispie_b200 import engine
    rng = np.random.default_rng(8)
    for ntr, nt in ((7, 1), (5, 256), (9, 1000), (3, 4097)):
        g = rng.standard_normal((ntr, nt)).astype(np.float32)
        want = np.flip(np.cumsum(np.flip(g.astype(np.float64), -1), -1), -1)
        gt = torch.as_tensor(g).cuda()
        out = engine.trace_suffix_sum(gt)
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-6, atol=1e-5)
        engine.trace_suffix_sum(gt, gt)  # in place
        assert torch.equal(gt, out)


def _wide_case(mode, nshots=11, nrec=300, nx=70, nz=66, nt=200):
    """Several tiles, more shots than a cluster, more receivers than a CTA
    compacts at once, receivers on and next to tile edges."""
    from seispie_b200.adjoint import AcquisitionSetup
    from seispie_b200.engine import Grid
    setup, p, src, rec, absorb, rng = _case(mode, seed=11, nx=nx, nz=nz, nt=nt)
    h = setup.grid.dx
    src = np.array([[h * (6 + 5 * s), h * (8 + (7 * s) % 50), 0, 14.0, 0.07 + 0.003 * s, 10.0 * s, 1e10]
                    for s in range(nshots)])
    xs = [30, 31, 32, 33, 34, 63, 64, 65, 2, 5, 47]
    rec = np.array([[h * xs[r % len(xs)], h * (3 + (r * 7) % (nz - 6))] for r in range(nrec)])
    setup = AcquisitionSetup(mode, Grid(nx, nz, h, h), setup.dt, nt, src, rec, absorb, segment=23)
    return setup, p, src, rec, absorb


@pytest.mark.parametrize("mode", ["sh", "psv"])
def test_exact_gradient_many_shots_tiles_receivers(mode):
    from seispie_b200.adjoint import AcquisitionSetup
    setup, p, src, rec, absorb = _wide_case(mode)
    data = _data(setup, p, src, absorb)
    grad, _ = _gpu_grad(setup, p, data)
    g = setup.grid
    i, j = np.meshgrid(np.arange(g.nx), np.arange(g.nz), indexing="ij")
    direction = {k: (0.5 + 0.5 * np.sin(0.17 * i + 0.11 * j + n)) * p[k] for n, k in enumerate(p)}
    eps = 1e-5
    pp = {k: p[k].astype(np.float64) + eps * direction[k] for k in p}
    pm = {k: p[k].astype(np.float64) - eps * direction[k] for k in p}
    fd = (_oracle_chi(setup, pp, src, absorb, data) - _oracle_chi(setup, pm, src, absorb, data)) / (2 * eps)
    dd = sum(float((grad[k] * direction[k]).sum()) for k in p)
    assert abs(dd - fd) < 1e-4 * abs(fd), (dd, fd)
    # the batched gradient is the sum of the one-shot gradients
    total = {k: np.zeros_like(v) for k, v in grad.items()}
    for s in range(len(src)):
        one = AcquisitionSetup(mode, g, setup.dt, setup.nt, src[s:s + 1], rec, absorb, segment=23)
        gs, _ = _gpu_grad(one, p, data[:, s:s + 1])
        for k in total:
            total[k] += gs[k]
    for k in grad:
        scale = np.abs(grad[k]).max()
        np.testing.assert_allclose(grad[k], total[k], rtol=0, atol=2e-5 * scale, err_msg=k)


def test_spin_exact_gradient_directional_derivatives():
    """Micropolar spin: the exact adjoint's gradient along a smooth direction
    of each of the seven parameters (rho, lam, mu, nu, j, mu_c, nu_c) against
    central finite differences of the FP64 oracle's misfit (x and z traces)."""
    from seispie_b200 import engine
    from seispie_b200.adjoint import AcquisitionSetup, ExactAdjoint, hann_taper
    from seispie_b200.engine import Grid, build_model
    nx, nz, nt, h, dt = 40, 36, 240, 10.0, 1e-3
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    sm = lambda a, b, c: np.sin(a * i / nx + b * j / nz + c)  # noqa: E731
    p = dict(rho=2700 * (1 + 0.03 * sm(1.7, 2.9, 2.0)), lam=8.1e9 * (1 + 0.05 * sm(3.1, 2.2, 0.3)),
             mu=8.1e9 * (1 + 0.04 * sm(2.3, 3.7, 1.1)), nu=1.005e9 * (1 + 0.05 * sm(1.3, 2.1, 0.7)),
             j=2700 * (1 + 0.05 * sm(2.9, 1.1, 0.2)), mu_c=1.5e8 * (1 + 0.05 * sm(1.9, 2.7, 1.4)),
             nu_c=3.0e8 * (1 + 0.05 * sm(0.9, 3.3, 2.5)))
    p = {k: v.astype(np.float32) for k, v in p.items()}
    src = np.array([[120.0, 150.0, 0, 14.0, 0.07, 25.0, 1e10], [260.0, 90.0, 0, 12.0, 0.08, -40.0, 1e10]])
    rec = np.array([[50.0 + 45 * r, 30.0 + 40 * (r % 3)] for r in range(6)])
    absorb = (8, 0.05, 1, 1, 1, 0)
    grid = Grid(nx, nz, h, h)
    setup = AcquisitionSetup("spin", grid, dt, nt, src, rec, absorb, segment=37)
    o = Oracle("f64")
    stf = source_time_functions(src, nt, dt)
    w = hann_taper(nt, dt) ** 2
    bound = o.set_bound(nx, nz, *absorb)
    nrec = len(setup.rec_id)

    def traces(q):
        out = []
        for s in range(setup.nshots):
            prm = dict(bound=bound, **{k: np.asarray(v, np.float64).ravel() for k, v in q.items()})
            obs, _, _ = o.forward("spin", nx, nz, h, h, dt, nt, prm, setup.src_id, stf, s, setup.rec_id)
            out.append([obs[c].reshape(-1, nt) for c in "xz"])
        return np.array(out)  # [shot, component, receiver, t]

    q = {k: v.astype(np.float64) for k, v in p.items()}
    q["mu"] = q["mu"] * (1 + 0.03 * np.cos(np.arange(nx * nz).reshape(nx, nz) * 0.37))
    data = traces(q)

    def chi(q):
        r = traces(q) - data
        return float((w * r * r).sum())

    m = build_model("spin", grid, dt, {k: v.ravel() for k, v in p.items()}, absorb, "cuda")
    ea = ExactAdjoint(m, nt, setup.src_id, setup.isrc_of_shot, setup.nshots, setup.stf, setup.rec_id, segment=37)
    tr = ea.forward()
    g = [None, None, None]
    for ci, c in enumerate((0, 2)):
        d = torch.as_tensor(np.ascontiguousarray(data[:, ci]).astype(np.float32), device="cuda").reshape(-1)
        g[c] = torch.empty(setup.nshots * nrec * nt, device="cuda")
        engine.misfit_tracegrad(d, tr[c].reshape(-1).contiguous(), g[c], setup.nshots, nrec, nt, dt)
        g[c] = g[c].view(setup.nshots, nrec, nt)
    k = ea.backward(g)
    dlam, dmu, dbuo, dnu, dmnc, dbuoj = (t[:, :nz].double().cpu().numpy() for t in k)
    grad = dict(lam=dlam, mu=dmu, nu=dnu, mu_c=dmnc, nu_c=dmnc,
                rho=-dbuo * dt / p["rho"].astype(np.float64) ** 2, j=-dbuoj * dt / p["j"].astype(np.float64) ** 2)
    eps = 1e-5
    for n, name in enumerate(("rho", "lam", "mu", "nu", "j", "mu_c", "nu_c")):
        direction = (0.5 + 0.5 * np.sin(0.21 * i + 0.13 * j + n)) * p[name].astype(np.float64)
        qp = {kk: v.astype(np.float64) for kk, v in p.items()}
        qm = {kk: v.astype(np.float64) for kk, v in p.items()}
        qp[name] = qp[name] + eps * direction
        qm[name] = qm[name] - eps * direction
        fd = (chi(qp) - chi(qm)) / (2 * eps)
        dd = float((grad[name] * direction).sum())
        assert abs(dd - fd) < 2e-3 * abs(fd), (name, dd, fd)


@pytest.mark.parametrize("mode", ["psv", "spin"])
def test_two_level_checkpointing_is_bit_identical(mode):
    """Recursive (two-level) checkpointing, per-step stores kept from the
    forward sweep for the last steps, and the backward that recomputes one
    segment ahead on a second stream produce the same forward values as
    single-level recomputation, so the gradients are equal exactly."""
    from seispie_b200.adjoint import AcquisitionSetup, ExactAdjoint
    from seispie_b200.engine import Grid, build_model
    nx, nz, nt, h, dt = 40, 36, 230, 10.0, 1e-3
    rng = np.random.default_rng(6)
    src = np.array([[120.0, 150.0, 0, 14.0, 0.07, 25.0, 1e10], [260.0, 90.0, 0, 12.0, 0.08, -40.0, 1e10]])
    rec = np.array([[50.0 + 45 * r, 30.0 + 40 * (r % 3)] for r in range(6)])
    absorb = (8, 0.05, 1, 1, 1, 0)
    grid = Grid(nx, nz, h, h)
    setup = AcquisitionSetup(mode, grid, dt, nt, src, rec, absorb)
    npt = nx * nz
    prm = dict(rho=np.full(npt, 2700.0), lam=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)),
               mu=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)))
    if mode == "spin":
        prm.update(nu=np.full(npt, 1.005e9), j=np.full(npt, 2700.0), mu_c=np.full(npt, 1.5e8), nu_c=np.full(npt, 3e8))
    m = build_model(mode, grid, dt, prm, absorb, "cuda")
    nrec = len(setup.rec_id)
    g = [torch.randn(setup.nshots, nrec, nt, device="cuda") if c != 1 else None for c in range(3)]
    # per-step stores kept from the forward sweep for the last 61 steps
    per_step = (6 + 3 if mode == "spin" else 3 + 2) * 4 * setup.nshots * nx * grid.pitch
    out = []
    for kw in (dict(segment=37), dict(levels=2, segment=50, sub_segment=7),
               dict(segment=37, tail_memory=61.5 * per_step), dict(segment=37, overlap=True),
               dict(segment=23, tail_memory=61.5 * per_step, overlap=True),
               dict(segment=37, tail_memory=61.5 * per_step * 6 / 9 if mode == "spin" else 61.5 * per_step * 3 / 5,
                    density=False)):
        ea = ExactAdjoint(m, nt, setup.src_id, setup.isrc_of_shot, setup.nshots, setup.stf, setup.rec_id, **kw)
        tr = ea.forward()
        out.append((tr, ea.backward(g), ea.illum.clone()))
        if "tail_memory" in kw:
            assert ea.tail == 61 and ea.t0 == nt - 61
        if not kw.get("density", True):  # no divergence stores, no buoyancy terms
            assert all(t is None for t in ea.seg_ds + ea.tail_ds)
            assert out[-1][1][2] is None and (mode != "spin" or out[-1][1][5] is None)
        assert ea.overlap == kw.get("overlap", False)
    (tr1, k1, il1) = out[0]
    assert len(k1) == (6 if mode == "spin" else 3)
    for tr2, k2, _ in out[1:]:
        for c in (0, 2):
            assert torch.equal(tr1[c], tr2[c])
        for a, b in zip(k1, k2):
            assert b is None or torch.equal(a, b)
    assert float(k1[1].abs().max()) > 0
    # the illumination is sampled at the multiples of the segment whether or not a stored tail
    # takes the last steps, so it does not depend on the memory the tail got
    assert torch.equal(il1, out[2][2]) and float(il1.max()) > 0


@pytest.mark.parametrize("nx,nz,nshots,nrec", [(70, 133, 5, 300), (96, 128, 3, 40), (33, 37, 1, 7), (64, 200, 9, 12)])
def test_psv_wide_tile_transposed_step_is_bit_identical(nx, nz, nshots, nrec):
    """The P-SV transposed step on 32 x 64 tiles (two z columns per thread,
    the default) against 32 x 32 tiles (one column per thread), from the
    same random adjoint state, segment stores and receiver injections: the
    adjoint fields agree bit for bit, the FP64 gradient terms to the
    rounding of their summation over a cluster's shots (the two tilings pick
    different cluster sizes).  Grids that are not multiples of the tiles, an
    odd nz, one shot, and more injection entries per shot than one CTA's
    list holds (300)."""
    from seispie_b200.engine import Grid, ShotBatch, adjoint_injection_lists, build_model
    rng = np.random.default_rng(nx * 1000 + nz)
    h, dt, nt, it = 10.0, 1e-3, 6, 3
    grid = Grid(nx, nz, h, h)
    npt = nx * nz
    prm = dict(rho=2600 * (1 + 0.05 * rng.random(npt)), lam=8.1e9 * (1 + 0.05 * rng.random(npt)),
               mu=8.1e9 * (1 + 0.05 * rng.random(npt)))
    m = build_model("psv", grid, dt, prm, (8, 0.05, 1, 1, 1, 0), "cuda")
    rec = rng.integers(0, npt, nrec).astype(np.int32)
    shape = (nshots, nx, grid.pitch)

    def field():
        t = torch.randn(shape, device="cuda")
        t[..., nz:] = 0.0  # padding cells stay zero
        return t

    state = [field() for _ in range(5)]
    seg_e = [field()[None] for _ in range(3)] + [None] * 3
    seg_ds = [field()[None], None, field()[None]]
    stf = [torch.randn(nshots * nrec * nt, device="cuda"), None, torch.randn(nshots * nrec * nt, device="cuda")]
    inj = adjoint_injection_lists(nshots, rec)
    out = []
    for tile in (0, 1):
        b = ShotBatch(m, nshots, nt, rec)
        b.adj_tile = tile
        for t, s in zip(b.sig[0] + b.vel[0], state):
            t.copy_(s)
        k = [torch.zeros((nx, grid.pitch), dtype=torch.float64, device="cuda") for _ in range(3)]
        d = b.desc(inj=inj, stf=stf, record=False, kernels=k)
        b.set_segment(d, seg_e, seg_ds, it, 1)
        b.run_transposed(d, it + 1, 1)
        torch.cuda.synchronize()
        assert d.cur == 1
        out.append(([t.clone() for t in b.sig[1] + b.vel[1]], k))
    (f0, k0), (f1, k1) = out
    for a, c in zip(f0, f1):
        assert float(a.abs().max()) > 0
        assert torch.equal(a, c)
    for a, c in zip(k0, k1):
        scale = float(c.abs().max())
        assert scale > 0 and float((a - c).abs().max()) <= 1e-6 * scale


@pytest.mark.parametrize("mode", ["sh", "psv"])
def test_step_overlap_is_bit_identical(mode):
    """Programmatic dependent launch between the steps of a time loop
    (fwi_batch.step_overlap, the default) against serialised launches: the
    row-marching forward and recomputed steps and the wide-tile transposed
    steps read the previous step only after it has completed, so traces,
    every gradient term and the illumination agree bit for bit.  Checkpoint
    segments and a stored tail, with the serial backward (early launches in
    both kernels) and the overlapped one (none on its two streams)."""
    from seispie_b200.adjoint import AcquisitionSetup, ExactAdjoint
    from seispie_b200.engine import Grid, build_model
    nx, nz, nt, h, dt = 96, 130, 240, 10.0, 1e-3
    rng = np.random.default_rng(11)
    src = np.array([[120.0 + 150 * s, 150.0 + 70 * (s % 3), 0, 14.0, 0.07, 25.0, 1e10] for s in range(4)])
    rec = np.array([[50.0 + 37 * r, 30.0 + 40 * (r % 3)] for r in range(23)])
    absorb = (8, 0.05, 1, 1, 1, 0)
    grid = Grid(nx, nz, h, h)
    setup = AcquisitionSetup(mode, grid, dt, nt, src, rec, absorb)
    npt = nx * nz
    prm = dict(rho=np.full(npt, 2700.0) * (1 + 0.05 * rng.random(npt)),
               lam=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)),
               mu=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)))
    m = build_model(mode, grid, dt, prm, absorb, "cuda")
    nrec = len(setup.rec_id)
    # trace gradients of the recorded components (SH: y; P-SV: x and z)
    g = [torch.randn(setup.nshots, nrec, nt, device="cuda") if (c == 1) == (mode == "sh") else None
         for c in range(3)]
    per_step = 5 * 4 * setup.nshots * nx * grid.pitch
    out = []
    for on, overlap in ((True, False), (False, False), (True, True), (False, True)):
        ea = ExactAdjoint(m, nt, setup.src_id, setup.isrc_of_shot, setup.nshots, setup.stf, setup.rec_id,
                          segment=23, tail_memory=41.5 * per_step, overlap=overlap, step_overlap=on)
        assert ea.fdesc.step_overlap == int(on)
        tr = ea.forward()
        k = ea.backward(g)
        torch.cuda.synchronize()
        out.append(([t.clone() if t is not None else None for t in tr], k, ea.illum.clone()))
    tr1, k1, il1 = out[0]
    assert any(t is not None and float(t.abs().max()) > 0 for t in tr1)
    assert float(k1[1].abs().max()) > 0  # dL/dmu (dL/dlam is zero for SH)
    for tr2, k2, il2 in out[1:]:
        for a, b in zip(tr1, tr2):
            assert (a is None and b is None) or torch.equal(a, b)
        for a, b in zip(k1, k2):
            assert (a is None and b is None) or torch.equal(a, b)
        assert torch.equal(il1, il2)


@pytest.mark.parametrize("overlap", [False, True])
def test_gradient_graph_is_bit_identical(overlap):
    """One exact gradient (forward sweep, misfit and trace gradients,
    backward) captured in one CUDA graph and replayed: traces, misfit,
    every gradient term and the illumination equal the eager run's bit for
    bit, on two replays in a row and again after the model tensors have been
    changed in place (the graph reads the model's current values)."""
    from seispie_b200 import engine
    from seispie_b200.adjoint import AcquisitionSetup, ExactAdjoint, GradientGraph
    from seispie_b200.engine import Grid, build_model
    nx, nz, nt, h, dt = 96, 130, 240, 10.0, 1e-3
    rng = np.random.default_rng(12)
    src = np.array([[120.0 + 150 * s, 150.0 + 70 * (s % 3), 0, 14.0, 0.07, 25.0, 1e10] for s in range(4)])
    rec = np.array([[50.0 + 37 * r, 30.0 + 40 * (r % 3)] for r in range(23)])
    absorb = (8, 0.05, 1, 1, 1, 0)
    grid = Grid(nx, nz, h, h)
    setup = AcquisitionSetup("psv", grid, dt, nt, src, rec, absorb)
    npt = nx * nz
    prm = dict(rho=np.full(npt, 2700.0) * (1 + 0.05 * rng.random(npt)),
               lam=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)),
               mu=np.full(npt, 8.1e9) * (1 + 0.05 * rng.random(npt)))
    m = build_model("psv", grid, dt, prm, absorb, "cuda")
    nrec, ns = len(setup.rec_id), setup.nshots
    data = [torch.randn(ns * nrec * nt, device="cuda") * 1e-9 if c != 1 else None for c in range(3)]
    grads = [torch.empty((ns, nrec, nt), device="cuda") if c != 1 else None for c in range(3)]
    per_step = 3 * 4 * ns * nx * grid.pitch

    def make():
        return ExactAdjoint(m, nt, setup.src_id, setup.isrc_of_shot, ns, setup.stf, setup.rec_id, segment=23,
                            tail_memory=41.5 * per_step, overlap=overlap, density=False)

    def between(tr):
        mis = [engine.misfit_tracegrad(data[c], tr[c].reshape(-1), grads[c], ns, nrec, nt, dt) for c in (0, 2)]
        return grads, torch.stack(mis)

    def eager():
        ea = make()
        tr = ea.forward()
        g, mis = between(tr)
        k = ea.backward(g)
        torch.cuda.synchronize()
        return [t.clone() if t is not None else None for t in tr], mis.clone(), k, ea.illum.clone()

    def same(x, y):
        (tr1, m1, k1, i1), (tr2, m2, k2, i2) = x, y
        for a, b in zip(tr1, tr2):
            assert (a is None and b is None) or torch.equal(a, b)
        assert torch.equal(m1, m2)
        for a, b in zip(k1, k2):
            assert (a is None and b is None) or torch.equal(a, b)
        assert torch.equal(i1, i2)

    ref = eager()
    assert float(ref[2][1].abs().max()) > 0 and float(ref[1].sum()) > 0
    gg = GradientGraph(make(), between)
    assert gg.launches > 2 * nt  # every forward, recomputed and transposed step is a node
    for _ in range(2):
        tr, mis, k = gg.replay()
        torch.cuda.synchronize()
        same(ref, ([t.clone() if t is not None else None for t in tr], mis.clone(), k, gg.illum.clone()))
    m.mu.mul_(1.02)
    m.lam.mul_(0.99)
    ref2 = eager()
    assert not torch.equal(ref2[2][1], ref[2][1])
    tr, mis, k = gg.replay()
    torch.cuda.synchronize()
    same(ref2, ([t.clone() if t is not None else None for t in tr], mis.clone(), k, gg.illum.clone()))


def _psv_plugin(root, **over):
    """A b200 plugin on a small P-SV checkerboard case (observed traces
    imported from the true model, the initial model loaded)."""
    import os
    from seispie_b200.io import write_model
    from seispie_b200.solver import b200
    nx, nz, h, nt = 44, 38, 10.0, 240
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    vs_true = 1732 * (1 + 0.05 * np.sign(np.sin(i / 5.0) * np.sin(j / 5.0) + 1e-9))
    for d, vs in (("true", vs_true.ravel()), ("init", np.full(nx * nz, 1732.0))):
        if not os.path.isdir(os.path.join(root, d)):
            write_model(os.path.join(root, d), nx, nz, h, h, dict(vp=np.full(nx * nz, 3000.0), vs=vs,
                                                                  rho=np.full(nx * nz, 2600.0)))
    src = np.array([[100.0, 60.0, 0, 14.0, 0.07, 20.0, 1e10], [300.0, 60.0, 0, 14.0, 0.07, -30.0, 1e10],
                    [200.0, 90.0, 0, 14.0, 0.07, 10.0, 1e10]])
    rec = np.array([[30.0 + 30 * r, 80.0] for r in range(12)])
    np.savetxt(os.path.join(root, "src.dat"), src)
    np.savetxt(os.path.join(root, "rec.dat"), rec)
    os.makedirs(os.path.join(root, "out"), exist_ok=True)
    s = b200()
    s.config = dict(nt=str(nt), dt="1e-3", sh="no", psv="yes", abs_left="yes", abs_right="yes", abs_top="no",
                    abs_bottom="yes", abs_width="8", abs_alpha="0.05", save_coordinates="", combine_sources="no",
                    save_snapshot="0", adjoint_interval="4", smooth="2")
    s.config.update(over)
    s.path = dict(model_true=os.path.join(root, "true"), model_init=os.path.join(root, "init"),
                  sources=os.path.join(root, "src.dat"), stations=os.path.join(root, "rec.dat"),
                  output=os.path.join(root, "out"))
    s.mpi = None
    s.setup(None)
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.import_traces()
    s.import_model(0)
    return s


def test_plugin_gradient_graph_replays_bit_identical(tmp_path):
    """compute_gradient of the plugin keeps the exact gradient of its shots
    in a CUDA graph after the first call and replays it on the next ones:
    misfits and the FP64 lambda / mu kernels equal those of a plugin that
    never captures (cuda_graph = no) bit for bit, over three gradients with
    the model changed in place between them; a new model drops the graph."""
    a = _psv_plugin(str(tmp_path))
    b = _psv_plugin(str(tmp_path), cuda_graph="no")
    npt = a.nx * a.nz
    rng = np.random.default_rng(5)
    for it in range(3):
        ra = a.compute_gradient()
        rb = b.compute_gradient()
        assert ra[1] == rb[1] and ra[1] > 0  # misfit
        for k in ("k_lam_f64", "k_mu_f64"):
            assert torch.equal(getattr(a, k), getattr(b, k)), (it, k)
        assert np.array_equal(ra[0], rb[0])  # smoothed kernel
        assert len(a._graphs) == 1 and not getattr(b, "_graphs", None)
        new_mu = ((2600.0 * 1732.0 ** 2) * (1 + 0.01 * (it + 1) * rng.standard_normal(npt))).astype(np.float32)
        a.update_model(new_mu)
        b.update_model(new_mu)
    a.import_model(0)
    assert not a._graphs
