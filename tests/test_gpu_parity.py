"""Parity of the CUDA path (through the C-ABI) with the reference's golden
vectors and with the CPU oracle.

Tolerances (relative L2): seismograms 1e-5, sensitivity kernels 1e-4, as the
solver's accuracy target states; integer work (point ids) and the float32
set-up kernels written with explicit rounding (vps2lm, set_bound, misfit
adjoint source) are compared bit for bit.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle.oracle import Oracle, point_ids, source_time_functions  # noqa: E402
from tests.conftest import load_golden  # noqa: E402
from tests.gpu_helpers import make_model, rel, run_forward, state, traces  # noqa: E402

TRACE_TOL = 1e-5
KERNEL_TOL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from seispie_b200 import _lib
    _lib.load()


def golden_model(g):
    mode, nx, nz = str(g["mode"]), int(g["nx"]), int(g["nz"])
    cfg = eval(str(g["config"]))
    absorb = (int(cfg["abs_width"]), float(cfg["abs_alpha"]), cfg["abs_left"] == "yes", cfg["abs_right"] == "yes",
              cfg["abs_bottom"] == "yes", cfg["abs_top"] == "yes")
    if mode == "spin":
        params = dict(rho=g["model_rho"], lam=g["model_lambda"], mu=g["model_mu"], nu=g["model_nu"],
                      j=g["model_j"], mu_c=g["model_mu_c"], nu_c=g["model_nu_c"])
    else:
        params = dict(rho=g["model_rho"], vp=g["model_vp"], vs=g["model_vs"])
    return mode, nx, nz, make_model(mode, nx, nz, g["dx"], g["dz"], float(g["dt"]), params, absorb), params, absorb


@pytest.mark.parametrize("name", ["sh_fwd", "psv_fwd"])
def test_model_setup_bit_exact(name):
    g = load_golden(name)
    mode, nx, nz, m, _, _ = golden_model(g)
    un = lambda t: t[:, :nz].reshape(-1).cpu().numpy()  # noqa: E731
    assert np.array_equal(un(m.lam), g["lam"])
    assert np.array_equal(un(m.mu), g["mu"])
    assert np.array_equal(un(m.bound), g["bound"])


def test_ricker_matches_reference():
    from seispie_b200 import engine
    g = load_golden("example_geometry")
    stf, _ = engine.ricker_stf(g["src"][:2], int(g["nt"]), float(g["dt"]), "cuda")
    got = stf[1].cpu().numpy()
    ref = g["stf_y01"]
    ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1  # FP64 exp of CUDA vs numpy, rounded to float32
    assert rel(got, ref) < 1e-7


@pytest.mark.parametrize("name,displacement", [("sh_fwd", True), ("sh_fwd", False), ("sh_fwd_task1", True),
                                                ("sh_fwd_task1", False), ("psv_fwd", True), ("psv_fwd", False),
                                                ("spin_fwd", True)])
def test_forward_matches_reference_golden(name, displacement):
    """Traces and final wavefields against the reference run, with the tiled
    kernel and displacement fields, and displacement-free (row-marching
    kernel; no displacement field to compare)."""
    g = load_golden(name)
    mode, nx, nz, m, _, _ = golden_model(g)
    sid = point_ids(g["src"], g["dx"], g["dz"], nz)
    rid = point_ids(g["rec"], g["dx"], g["dz"], nz)
    b = run_forward(m, int(g["nt"]), g["src"], sid, rid, [int(g["isrc"])], displacement=displacement)
    comps = {"x": 0, "y": 1, "z": 2}
    for c, ci in comps.items():
        if "obs_" + c in g:
            assert rel(traces(b, ci)[0], g["obs_" + c]) < TRACE_TOL, c
    for k in g:
        if k.startswith("state_") and (displacement or not k.startswith("state_u")):
            assert rel(state(b, k[6:])[0], g[k]) < TRACE_TOL, k


def _march_vs_tiled(mode, nx, nz, isrcs, nt, seed, chunks=None, src=None, rec=None):
    """Run one case displacement-free (row-marching kernel) and with
    displacement fields (tiled kernel); assert traces, stress and velocity
    are equal bit for bit."""
    params, src0, rec0, absorb, h, dt, _ = _medium_case(mode, seed, nx, nz)
    src = src0 if src is None else src
    rec = rec0 if rec is None else rec
    m = make_model(mode, nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    ref = run_forward(m, nt, src, sid, rid, isrcs, displacement=True)
    got = run_forward(m, nt, src, sid, rid, isrcs, displacement=False, chunks=chunks)
    comps = [1] if mode == "sh" else [0, 2]
    for c in comps:
        t = traces(got, c)
        assert np.abs(t).max() > 0
        assert np.array_equal(t, traces(ref, c)), c
    names = ("vy", "sxy", "szy") if mode == "sh" else ("vx", "vz", "sxx", "szz", "sxz")
    for f in names:
        assert np.array_equal(state(got, f), state(ref, f)), f


@pytest.mark.parametrize("mode", ["sh", "psv"])
@pytest.mark.parametrize("nx,nz,nshots", [(83, 70, 3), (61, 45, 2), (9, 1021, 1), (130, 20, 5), (5, 64, 2)])
def test_displacement_free_bit_identical(mode, nx, nz, nshots):
    """The row-marching kernel does the tiled kernels' arithmetic per cell,
    and the traces rebuilt from the velocity at the receivers equal the
    displacement the tiled kernels keep: bit for bit, on grids with nz not a
    multiple of 4, nz near the 1024-column limit, a 5-row grid, more shots
    than sources (isrc -1: all of them), the time loop in several calls."""
    isrcs = [(-1 if s % 3 == 2 else s % 3) for s in range(nshots)]
    h = 10.0
    # sources and receivers spread over the grid, receivers a few cells from the sources
    src = np.array([[(nx // 2) * h, (nz // 3) * h, 0, 12.0, 0.08, 30.0, 1e10],
                    [(nx // 3) * h, (nz // 2) * h, 0, 10.0, 0.1, -60.0, 1e10],
                    [(nx - 1) * h, 2 * h, 0, 14.0, 0.07, 0.0, 1e10]])
    rec = np.array([[0, 0], [(nx - 1) * h, (nz - 1) * h], [0, (nz - 1) * h], [(nx - 1) * h, 5 * h]] +
                   [[min(nx - 1, nx // 2 + d) * h, min(nz - 1, nz // 3 + 3 * d) * h] for d in range(4)] +
                   [[(nx // 3) * h, min(nz - 1, nz // 2 + d) * h] for d in (-2, 1, 4)])
    _march_vs_tiled(mode, nx, nz, isrcs, 70, seed=nx + nz, chunks=[1, 23, 46], src=src, rec=rec)


def test_displacement_free_bit_identical_full_size():
    """512 x 512, 32 shots (every CTA marches tens of rows and the shots'
    row ranges split across CTAs), 256 receivers in a line, 25 steps."""
    nx = nz = 512
    h = 10.0
    src = np.array([[(s + 0.5) * nx / 32 * h, 10 * h, 0, 8.0, 0.15, 0.0, 1e10] for s in range(32)])
    rec = np.array([[(r + 0.5) * nx / 256 * h, 12 * h] for r in range(256)])
    _march_vs_tiled("psv", nx, nz, list(range(32)), 25, seed=1, src=src, rec=rec)


@pytest.mark.parametrize("mode", ["sh", "psv"])
def test_displacement_free_many_points(mode):
    """More sources and receivers in a CTA's rows than its shared-memory
    windows hold (256), several on one cell: the windows are refilled
    during the march and same-cell sources add in entry order."""
    nx, nz = 12, 48
    rng = np.random.default_rng(4)
    h = 10.0
    cells = rng.integers(0, nx * nz, 700)
    src = np.array([[(c // nz) * h, (c % nz) * h, 0, 10.0 + (c % 5), 0.1, 15.0 * (c % 7), 1e9 * (1 + c % 3)]
                    for c in cells])
    rec = np.array([[(c // nz) * h, (c % nz) * h] for c in rng.integers(0, nx * nz, 600)])
    _march_vs_tiled(mode, nx, nz, [-1, -1], 40, seed=2, src=src, rec=rec)


def _medium_case(mode, seed, nx=83, nz=70, nt=300, nsrc=3, nrec=9):
    rng = np.random.default_rng(seed)
    h, dt = 10.0, 1e-3
    n = nx * nz
    if mode == "spin":
        h, dt = 2.0, 2e-4
        base = dict(rho=2700.0, lam=8.1e9, mu=8.1e9, nu=10.05e8, j=2700.0, mu_c=1.5e8, nu_c=3.0e8)
        params = {k: (v * (1 + 0.05 * rng.uniform(-1, 1, n))).astype(np.float32) for k, v in base.items()}
    else:
        params = dict(vp=(3000 + 300 * rng.uniform(-1, 1, n)).astype(np.float32),
                      vs=(1732 + 200 * rng.uniform(-1, 1, n)).astype(np.float32),
                      rho=(2600 + 200 * rng.uniform(-1, 1, n)).astype(np.float32))
    f0 = 10.0 if mode != "spin" else 60.0
    src = np.array([[rng.uniform(3, max(4, nx - 4)) * h, rng.uniform(3, max(4, nz - 4)) * h, 0, f0, 1.2 / f0,
                     rng.uniform(-90, 90), 1e10] for _ in range(nsrc)])
    # receivers include the grid's edge rows and columns
    rec = np.array([[0, 0], [(nx - 1) * h, (nz - 1) * h], [0, (nz - 1) * h], [(nx - 1) * h, 5 * h]] +
                   [[rng.uniform(0, nx - 1) * h, rng.uniform(0, nz - 1) * h] for _ in range(nrec - 4)])
    absorb = (10, 0.04, 1, 1, 1, 0)
    return params, src, rec, absorb, h, dt, nt


def _oracle_forward(prec, mode, nx, nz, h, dt, nt, params, absorb, sid, src, rid, isrc, sae=0, snapshots=False):
    o = Oracle(prec)
    p = dict(params)
    if mode != "spin":
        p["lam"], p["mu"] = o.vps2lm(params["vp"], params["vs"], params["rho"])
    w, a, l, r, b, t = absorb
    p["bound"] = o.set_bound(nx, nz, w, a, l, r, b, t)
    stf = source_time_functions(src, nt, dt)
    return o, p, o.forward(mode, nx, nz, h, h, dt, nt, p, sid, stf, isrc, rid, sae=sae,
                           nsa=nt // sae if sae else 0, snapshots=snapshots)


@pytest.mark.parametrize("mode", ["sh", "psv", "spin"])
def test_forward_batched_vs_fp64_oracle(mode):
    """3 shots (one source each) in one batch on an 83x70 grid (nz not a
    multiple of 4: row padding; partial tiles), receivers on the edges."""
    nx, nz = 83, 70
    params, src, rec, absorb, h, dt, nt = _medium_case(mode, 7, nx, nz)
    m = make_model(mode, nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    b = run_forward(m, nt, src, sid, rid, [0, 1, 2])
    comps = {"sh": [1], "psv": [0, 2], "spin": [0, 2, 1]}[mode]
    for s in range(3):
        _, _, (obs, st, _) = _oracle_forward("f64", mode, nx, nz, h, dt, nt, params, absorb, sid, src, rid, s)
        for c in comps:
            assert rel(traces(b, c)[s], obs["xyz"[c]]) < TRACE_TOL, (s, c)
        for f in {"sh": ["vy", "sxy"], "psv": ["vx", "uz", "sxz"], "spin": ["vy_c", "syy_c", "szz"]}[mode]:
            assert rel(state(b, f)[s], st[f]) < TRACE_TOL, (s, f)


@pytest.mark.parametrize("mode", ["sh", "psv", "spin"])
def test_tile_variants_bit_identical(mode):
    """Every tile shape does the same arithmetic per cell."""
    from seispie_b200._lib import tile_variants
    nx, nz = 61, 45
    params, src, rec, absorb, h, dt, nt = _medium_case(mode, 3, nx, nz, nt=80)
    m = make_model(mode, nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    ref = run_forward(m, nt, src, sid, rid, [-1, 1], tile=0)
    for t in tile_variants():
        b = run_forward(m, nt, src, sid, rid, [-1, 1], tile=t)
        for f in ("uy", "sxy") if mode == "sh" else ("ux", "sxz"):
            assert np.array_equal(state(b, f), state(ref, f)), (t, f)


def test_batch_and_chunking_bit_identical():
    """A shot gives the same bits alone, in a batch, and with the time loop
    split across several fwi_run calls."""
    nx, nz = 50, 64
    params, src, rec, absorb, h, dt, nt = _medium_case("psv", 5, nx, nz, nt=90)
    m = make_model("psv", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    batch = run_forward(m, nt, src, sid, rid, [0, 1, 2])
    for s in range(3):
        one = run_forward(m, nt, src, sid, rid, [s], chunks=[1, 30, 17, 42])
        assert np.array_equal(traces(one, 0)[0], traces(batch, 0)[s])
        assert np.array_equal(state(one, "szz")[0], state(batch, "szz")[s])


def test_duplicate_sources_and_combined():
    """Two sources on one cell (combine_sources = yes): both add in entry
    order, as the reference's scatter does."""
    nx, nz, h, dt, nt = 40, 36, 10.0, 1e-3, 120
    params, _, rec, absorb, _, _, _ = _medium_case("sh", 9, nx, nz)
    src = np.array([[150.0, 170.0, 0, 12.0, 0.08, 0.0, 1e10], [150.0, 170.0, 0, 9.0, 0.1, 0.0, -4e9],
                    [60.0, 90.0, 0, 10.0, 0.1, 0.0, 2e9]])
    m = make_model("sh", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    b = run_forward(m, nt, src, sid, rid, [-1])
    _, _, (obs, _, _) = _oracle_forward("f64", "sh", nx, nz, h, dt, nt, params, absorb, sid, src, rid, -1)
    assert rel(traces(b, 1)[0], obs["y"]) < TRACE_TOL


def test_snapshots_match_oracle():
    """Forward snapshots (slot nsa-(it+1)/sae holds u before step it,
    solver.py:193-203), including a snapshot at a fwi_run chunk boundary."""
    nx, nz = 40, 44
    params, src, rec, absorb, h, dt, _ = _medium_case("psv", 4, nx, nz)
    nt, sae = 60, 7  # nt not a multiple of sae: the last steps store nothing
    m = make_model("psv", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    b = run_forward(m, nt, src, sid, rid, [1], sae=sae, snapshots=True, snap_velocity=True, chunks=[13, 20, 27])
    _, _, (_, _, sn) = _oracle_forward("f64", "psv", nx, nz, h, dt, nt, params, absorb, sid, src, rid, 1,
                                       sae=sae, snapshots=True)
    for c, slot in (("ux", 0), ("uz", 2)):
        got = b.snap_u[slot][:, 0, :, :nz].reshape(nt // sae, -1).cpu().numpy()
        assert rel(got, sn[c]) < TRACE_TOL, c
    for c, slot in (("vx", 0), ("vz", 2)):
        got = b.snap_v[slot][:, 0, :, :nz].reshape(nt // sae, -1).cpu().numpy()
        assert rel(got, sn[c]) < TRACE_TOL, c


def test_misfit_adjoint_source_golden():
    from seispie_b200 import engine
    g = load_golden("misfit_smooth")
    nt, nrec = int(g["nt"]), int(g["nrec"])
    data = torch.as_tensor(g["data"]).cuda()
    syn = torch.as_tensor(g["syn"]).cuda()
    adstf = torch.empty(nt * nrec, device="cuda")
    mis = engine.misfit(data, syn, adstf, 1, nrec, nt, float(g["dt"]))
    assert np.array_equal(adstf.cpu().numpy(), g["adstf"])
    assert abs(float(mis[0]) / float(g["misfit"]) - 1) < 1e-6


def test_smoothing_golden():
    from seispie_b200 import engine
    from seispie_b200.engine import Grid
    g = load_golden("misfit_smooth")
    nx, nz = int(g["nx"]), int(g["nz"])
    grid = Grid(nx, nz, 5.0, 5.0)
    k = torch.zeros((nx, grid.pitch), dtype=torch.float64, device="cuda")
    k[:, :nz] = torch.as_tensor(g["smooth_in"].astype(np.float64)).view(nx, nz)
    out = engine.smooth(k, grid, int(g["sigma"])).cpu().numpy()
    assert rel(out, g["smooth_out"]) < 1e-5


def test_smoothing_vs_oracle_large_sigma():
    """sigma large against the grid: the truncated sum equals the full one."""
    from seispie_b200 import engine
    from seispie_b200.engine import Grid
    nx, nz, sigma = 70, 33, 9
    rng = np.random.default_rng(2)
    raw = rng.standard_normal(nx * nz)
    grid = Grid(nx, nz, 1.0, 1.0)
    k = torch.zeros((nx, grid.pitch), dtype=torch.float64, device="cuda")
    k[:, :nz] = torch.as_tensor(raw).view(nx, nz)
    out = engine.smooth(k, grid, sigma).cpu().numpy()
    ref = Oracle("f64").smooth(raw, nx, nz, sigma)
    assert rel(out, ref) < 1e-6


def test_sh_gradient_plugin_matches_reference(tmp_path):
    """The whole adjoint workflow through the plugin (import_traces,
    compute_gradient) against the reference's k_mu and misfit."""
    from tests.test_plugin_host import make_case_dir
    from seispie_b200.solver import b200
    g = load_golden("sh_grad")
    d = make_case_dir(tmp_path, g)
    s = b200()
    s.config = dict(eval(str(g["config"])))
    s.path = d
    s.mpi = None
    s.setup(None)
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.import_traces()
    for i in range(2):
        assert rel(s.syn_y[i], g["data"][i]) < TRACE_TOL
    s.import_model(0)
    k, misfit, mu = s.compute_gradient()
    assert np.array_equal(mu, g["mu"])
    assert abs(misfit / float(g["misfit"]) - 1) < 1e-5
    assert rel(k, g["k_mu"]) < KERNEL_TOL
    raw = s.k_mu_f64[:, : s.nz].reshape(-1).cpu().numpy()
    assert rel(raw, g["k_mu_raw"]) < KERNEL_TOL


def test_psv_adjoint_kernels_vs_oracle():
    """P-SV adjoint (defined by this project; the reference's branch cannot
    run) against the FP64 oracle restatement: k_lam, k_mu, k_rho."""
    from seispie_b200 import engine
    from seispie_b200.engine import adjoint_injection_lists
    nx, nz = 48, 40
    params, src, rec, absorb, h, dt, _ = _medium_case("psv", 11, nx, nz, nrec=8)
    nt, sae = 120, 4
    m = make_model("psv", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    isrcs = [0, 2]
    b = run_forward(m, nt, src, sid, rid, isrcs, sae=sae, snapshots=True, snap_velocity=True)
    rng = np.random.default_rng(1)
    nrec = len(rid)
    adstf = [torch.as_tensor(rng.standard_normal(len(isrcs) * nrec * nt).astype(np.float32)).cuda()
             if c != 1 else None for c in range(3)]
    k = [torch.zeros((nx, m.grid.pitch), dtype=torch.float64, device="cuda") for _ in range(3)]
    d = b.desc(inj=adjoint_injection_lists(len(isrcs), rid), stf=adstf, record=False, kernels=k)
    b.clear()
    b.run(d, True, 0, nt)
    o = Oracle("f64")
    kl, km, kr = (np.zeros(nx * nz) for _ in range(3))
    for q, s in enumerate(isrcs):
        _, p, (_, _, sn) = _oracle_forward("f64", "psv", nx, nz, h, dt, nt, params, absorb, sid, src, rid, s,
                                           sae=sae, snapshots=True)
        ax = adstf[0].cpu().numpy().reshape(len(isrcs), -1)[q]
        az = adstf[2].cpu().numpy().reshape(len(isrcs), -1)[q]
        o.adjoint_psv(nx, nz, h, h, dt, nt, p, rid, ax, az, sae, sn, kl, km, kr)
    for got, ref in zip(k, (kl, km, kr)):
        assert rel(got[:, :nz].reshape(-1).cpu().numpy(), ref) < KERNEL_TOL


def _plugin_case(tmp_path, g, **over):
    """The b200 plugin set up on the sh_grad golden geometry (config keys in
    `over` replaced), observed traces generated from the true model."""
    from tests.test_plugin_host import make_case_dir
    from seispie_b200.solver import b200
    s = b200()
    s.config = dict(eval(str(g["config"])), **over)
    s.path = make_case_dir(tmp_path, g)
    s.mpi = None
    s.setup(None)
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.import_traces()
    s.import_model(0)
    return s


def test_sh_run_adjoint_per_shot_matches_reference(tmp_path):
    """The reference's own per-shot loop (run_kernel, solver.py:343-365):
    taskid, run_forward, _compute_misfit, run_adjoint for each source, then
    the raw k_mu and the summed misfit against the reference's."""
    g = load_golden("sh_grad")
    s = _plugin_case(tmp_path, g)
    s.setup_adjoint()
    s.clear_kernels()
    misfit = 0.0
    for i in range(s.nsrc):
        s.taskid = i
        s.run_forward()
        misfit += s._compute_misfit("y", s.syn_y[i])
        s.run_adjoint()
    raw = s.k_mu_f64[:, : s.nz].reshape(-1).cpu().numpy()
    assert rel(raw, g["k_mu_raw"]) < KERNEL_TOL
    assert abs(misfit / float(g["misfit"]) - 1) < 1e-5


def test_psv_run_adjoint_per_shot_equals_batched_gradient(tmp_path):
    """P-SV through the per-shot protocol (exact transposed step; the
    reference's P-SV adjoint cannot run) gives the batched exact gradient of
    run_kernel: k_lam, k_mu, k_rho and the misfit."""
    g = load_golden("sh_grad")
    s = _plugin_case(tmp_path / "a", g, sh="no", psv="yes", kernel_rho="yes")
    misfit_b = s.run_kernel(1)[0]
    batched = [k.clone() for k in (s.k_lam_f64, s.k_mu_f64, s.k_rho_f64)]
    # without kernel_rho no divergence is stored: the same lambda / mu kernels bit for bit, no rho kernel
    s2 = _plugin_case(tmp_path / "b", g, sh="no", psv="yes")
    assert s2.run_kernel(1)[0] == misfit_b
    assert torch.equal(s2.k_lam_f64, batched[0]) and torch.equal(s2.k_mu_f64, batched[1])
    assert float(s2.k_rho_f64.abs().max()) == 0
    s.setup_adjoint()
    s.clear_kernels()
    misfit = 0.0
    for i in range(s.nsrc):
        s.taskid = i
        s.run_forward()
        misfit += s._compute_misfit("x", s.syn_x[i]) + s._compute_misfit("z", s.syn_z[i])
        s.run_adjoint()
    for got, ref in zip((s.k_lam_f64, s.k_mu_f64, s.k_rho_f64), batched):
        assert float(ref.abs().max()) > 0
        assert rel(got.cpu().numpy(), ref.cpu().numpy()) < 1e-10
    assert abs(misfit / misfit_b - 1) < 1e-9
    with pytest.raises(RuntimeError, match="run_forward"):
        s.run_adjoint()  # consumed: a second adjoint needs a new forward
