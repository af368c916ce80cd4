"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures in tests/golden/ were made by tests/golden/make_golden.py, which
runs icui/seispie's own fd2d plugin under Numba's CUDA simulator.  In float32
("as-reference") mode the oracle repeats the reference's arithmetic, so every
comparison here is bit-exact except the misfit norm, which the reference
accumulates in float32 and the oracle in float64.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, grid_geometry, point_ids, source_time_functions
from tests.conftest import load_golden


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def setup_case(o, g):
    mode, nx, nz = str(g["mode"]), int(g["nx"]), int(g["nz"])
    cfg = eval(str(g["config"]))  # repr of a dict of strings written by make_golden.py
    if mode == "spin":
        params = {k: g["model_" + m] for k, m in (("rho", "rho"), ("lam", "lambda"), ("mu", "mu"), ("nu", "nu"),
                                                   ("j", "j"), ("mu_c", "mu_c"), ("nu_c", "nu_c"))}
    else:
        lam, mu = o.vps2lm(g["model_vp"], g["model_vs"], g["model_rho"])
        params = dict(rho=g["model_rho"], lam=lam, mu=mu)
    params["bound"] = o.set_bound(nx, nz, int(cfg["abs_width"]), float(cfg["abs_alpha"]), cfg["abs_left"] == "yes",
                                  cfg["abs_right"] == "yes", cfg["abs_bottom"] == "yes", cfg["abs_top"] == "yes")
    return mode, nx, nz, params


@pytest.mark.parametrize("name", ["sh_fwd", "sh_fwd_task1", "psv_fwd", "spin_fwd"])
def test_forward_bit_exact(name):
    g = load_golden(name)
    o = Oracle("f32")
    mode, nx, nz, params = setup_case(o, g)
    if mode != "spin":
        assert np.array_equal(params["lam"], g["lam"]) and np.array_equal(params["mu"], g["mu"])
    assert np.array_equal(params["bound"], g["bound"])
    stf = source_time_functions(g["src"], int(g["nt"]), float(g["dt"]))
    for s, k in zip(stf, ("stf_x", "stf_y", "stf_z")):
        assert np.array_equal(s, g[k])
    sid = point_ids(g["src"], g["dx"], g["dz"], nz)
    rid = point_ids(g["rec"], g["dx"], g["dz"], nz)
    assert np.array_equal(sid, g["src_id"]) and np.array_equal(rid, g["rec_id"])
    obs, st, _ = o.forward(mode, nx, nz, float(g["dx"]), float(g["dz"]), float(g["dt"]), int(g["nt"]), params,
                           sid, stf, int(g["isrc"]), rid)
    for c in "xyz":
        if "obs_" + c in g:
            assert np.array_equal(obs[c], g["obs_" + c]), c
    for k in g:
        if k.startswith("state_"):
            assert np.array_equal(st[k[6:]], g[k]), k


@pytest.mark.parametrize("name", ["sh_fwd", "psv_fwd", "spin_fwd"])
def test_forward_f64_close(name):
    """FP64 oracle vs the float32 reference: the float32 rounding budget."""
    g = load_golden(name)
    o = Oracle("f64")
    mode, nx, nz, params = setup_case(o, g)
    stf = source_time_functions(g["src"], int(g["nt"]), float(g["dt"]))
    sid = point_ids(g["src"], g["dx"], g["dz"], nz)
    rid = point_ids(g["rec"], g["dx"], g["dz"], nz)
    obs, _, _ = o.forward(mode, nx, nz, float(g["dx"]), float(g["dz"]), float(g["dt"]), int(g["nt"]), params,
                          sid, stf, int(g["isrc"]), rid)
    for c in "xyz":
        if "obs_" + c in g:
            assert rel(obs[c], g["obs_" + c]) < 1e-5


def _gradient(prec, g):
    o = Oracle(prec)
    nx, nz, nt, sae, sigma = (int(g[k]) for k in ("nx", "nz", "nt", "sae", "sigma"))
    dx, dz, dt = float(g["dx"]), float(g["dz"]), float(g["dt"])
    cfg = eval(str(g["config"]))
    stf = source_time_functions(g["src"], nt, dt)
    sid = point_ids(g["src"], g["dx"], g["dz"], nz)
    rid = point_ids(g["rec"], g["dx"], g["dz"], nz)
    bound = o.set_bound(nx, nz, int(cfg["abs_width"]), float(cfg["abs_alpha"]), 1, 1, 1, 0)
    vp = np.full(nx * nz, 3000.0, np.float32)
    rho = np.full(nx * nz, 2600.0, np.float32)
    lt, mt = o.vps2lm(vp, g["true_vs"], rho)
    li, mi = o.vps2lm(vp, np.full(nx * nz, 1732.0, np.float32), rho)
    k_mu = np.zeros(nx * nz, o.dt)
    misfit, data, adstfs = 0.0, [], []
    for i in range(len(sid)):
        obs, _, _ = o.forward("sh", nx, nz, dx, dz, dt, nt, dict(rho=rho, lam=lt, mu=mt, bound=bound), sid, stf, i, rid)
        data.append(obs["y"])
        obs, _, sn = o.forward("sh", nx, nz, dx, dz, dt, nt, dict(rho=rho, lam=li, mu=mi, bound=bound), sid, stf, i,
                               rid, sae=sae, nsa=nt // sae, snapshots=True)
        m, adstf, _ = o.misfit(data[-1], obs["y"], nt, dt, len(rid))
        misfit += m
        adstfs.append(adstf)
        o.adjoint_sh(nx, nz, dx, dz, dt, nt, dict(rho=rho, lam=li, mu=mi, bound=bound), rid, adstf, sae, sn["uy"], k_mu)
    return dict(mu=mi, data=data, adstf=adstfs, misfit=misfit, k_raw=k_mu, k=o.smooth(k_mu, nx, nz, sigma))


def test_sh_gradient_bit_exact():
    """Whole adjoint workflow: traces, adjoint sources, k_mu before and after
    smoothing (solver.py:332-404, fd2d.py:349-352)."""
    g = load_golden("sh_grad")
    r = _gradient("f32", g)
    assert np.array_equal(r["mu"], g["mu"])
    for i in range(2):
        assert np.array_equal(r["data"][i], g["data"][i])
        assert np.array_equal(r["adstf"][i], g["adstf"][i])
    assert np.array_equal(r["k_raw"], g["k_mu_raw"])
    assert np.array_equal(r["k"], g["k_mu"])
    assert abs(r["misfit"] / float(g["misfit"]) - 1) < 1e-6


def test_sh_gradient_f64_close():
    g = load_golden("sh_grad")
    r = _gradient("f64", g)
    assert rel(r["k"], g["k_mu"]) < 1e-4
    assert abs(r["misfit"] / float(g["misfit"]) - 1) < 1e-5


def test_misfit_and_smoothing_bit_exact():
    g = load_golden("misfit_smooth")
    o = Oracle("f32")
    m, adstf, _ = o.misfit(g["data"], g["syn"], int(g["nt"]), float(g["dt"]), int(g["nrec"]))
    assert np.array_equal(adstf, g["adstf"])
    assert abs(m / float(g["misfit"]) - 1) < 1e-6
    s = o.smooth(g["smooth_in"], int(g["nx"]), int(g["nz"]), int(g["sigma"]))
    assert np.array_equal(s, g["smooth_out"])


def test_example_geometry():
    """Grid inference and point mapping on the reference's own
    examples/forward set-up (201x201, 12 sources, 132 stations)."""
    g = load_golden("example_geometry")
    nx, nz = int(g["nx"]), int(g["nz"])
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    x = (i * 2400.0).ravel().astype(np.float32)
    z = (j * 2400.0).ravel().astype(np.float32)
    gx, gz, dx, dz = grid_geometry(x, z, np.int32(g["npt"]))
    assert (gx, gz) == (nx, nz) and dx == g["dx"] and dz == g["dz"]
    assert np.array_equal(point_ids(g["src"], dx, dz, nz), g["src_id"])
    assert np.array_equal(point_ids(g["rec"], dx, dz, nz), g["rec_id"])
    stf = source_time_functions(g["src"][:2], int(g["nt"]), float(g["dt"]))
    assert np.array_equal(stf[1], g["stf_y01"])
    o = Oracle("f32")
    assert np.array_equal(o.set_bound(nx, nz, 20, 0.015, 1, 1, 1, 0), g["bound"])


def test_round_half_even_points():
    """fd2d.py:132-133 rounds x/dx half-to-even (numpy round)."""
    pts = np.array([[25.0, 35.0], [15.0, 45.0]])
    ids = point_ids(pts, np.float32(10.0), np.float32(10.0), 100)
    assert list(ids) == [2 * 100 + 4, 2 * 100 + 4]
