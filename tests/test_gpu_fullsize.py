"""Parity at the stated configurations, over their full time loops.

Long FP32 time loops are where rounding drift would show, so these cases
run the configurations as stated -- SH 256 x 256 for 2000 steps, two P-SV
shots of the 512 x 512 gradient configuration for 4000 steps, a spin case
of 2000 steps, the uneven 48-instance batch at every instance's full nt --
and compare with the FP64 oracle (and the float32 oracle, which restates
the reference's own arithmetic).  The exact gradient at the full 512 x 512,
32-shot, nt 4000 size is checked by a central difference of the misfit.

Tolerances: traces within relative L2 1e-5 of the FP64 oracle (the
solver's accuracy target); the float32 oracle, itself rounded differently
from the CUDA path, within 1e-4; the directional derivative within 1e-3.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle.oracle import Oracle, point_ids, source_time_functions  # noqa: E402
from tests.gpu_helpers import make_model, rel, run_forward, traces  # noqa: E402

TRACE_TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from seispie_b200 import _lib
    _lib.load()


def _oracle_traces(prec, mode, nx, nz, h, dt, nt, params, absorb, src, rec, isrc):
    o = Oracle(prec)
    p = dict(params)
    if "vp" in p:
        p["lam"], p["mu"] = o.vps2lm(params["vp"], params["vs"], params["rho"])
    p["bound"] = o.set_bound(nx, nz, *absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    obs, _, _ = o.forward(mode, nx, nz, h, h, dt, nt, p, sid, source_time_functions(src, nt, dt), isrc, rid)
    return obs


def test_c1_sh_256_nt2000_vs_oracles():
    """SH forward exactly as the plain-forward configuration states it:
    256 x 256, h 10 m, vs 1732, rho 2600, dt 1e-3, nt 2000, one 10 Hz Ricker
    at the centre, 64 receivers on z = 20 cells, 20-cell sponge (left,
    right, bottom).  Row-marching (displacement-free) and tiled kernels
    agree bit for bit; both match the oracles over all 2000 steps."""
    nx = nz = 256
    h, dt, nt = 10.0, 1e-3, 2000
    n = nx * nz
    params = dict(vp=np.full(n, 3000.0, np.float32), vs=np.full(n, 1732.0, np.float32),
                  rho=np.full(n, 2600.0, np.float32))
    absorb = (20, 0.015, 1, 1, 1, 0)
    src = np.array([[128 * h, 128 * h, 0, 10.0, 1.2 / 10.0, 0.0, 1e10]])
    rec = np.array([[(r + 0.5) * nx / 64 * h, 20 * h] for r in range(64)])
    m = make_model("sh", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    free = traces(run_forward(m, nt, src, sid, rid, [0], displacement=False), 1)[0]
    tiled = traces(run_forward(m, nt, src, sid, rid, [0], displacement=True), 1)[0]
    assert np.array_equal(free, tiled)
    ref64 = _oracle_traces("f64", "sh", nx, nz, h, dt, nt, params, absorb, src, rec, 0)["y"]
    ref32 = _oracle_traces("f32", "sh", nx, nz, h, dt, nt, params, absorb, src, rec, 0)["y"]
    assert np.abs(ref64).max() > 0
    assert rel(free, ref64) < TRACE_TOL
    assert rel(free, ref32) < 1e-4


def _c2_case():
    """The 512 x 512 P-SV gradient configuration: vp 3000 / vs 1732 /
    rho 2600 with a +-5 % vs checkerboard in 32 x 32 squares, 32 Ricker
    sources (8 Hz) at z = 10 cells, 256 receivers at z = 12 cells."""
    nx = nz = 512
    h = 10.0
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    board = np.where(((i // 32) + (j // 32)) % 2 == 0, 1.0, -1.0)
    n = nx * nz
    params = dict(vp=np.full(n, 3000.0, np.float32), vs=(1732.0 * (1 + 0.05 * board)).ravel().astype(np.float32),
                  rho=np.full(n, 2600.0, np.float32))
    src = np.array([[(s + 0.5) * nx / 32 * h, 10 * h, 0, 8.0, 1.2 / 8.0, 0.0, 1e10] for s in range(32)])
    rec = np.array([[(r + 0.5) * nx / 256 * h, 12 * h] for r in range(256)])
    return nx, nz, h, 1e-3, params, (20, 0.015, 1, 1, 1, 0), src, rec


def test_c2_two_shots_nt4000_vs_fp64():
    """Shots 0 and 31 of the 512 x 512 gradient configuration (the sources
    nearest the two side sponges), batched, all 4000 steps."""
    nx, nz, h, dt, params, absorb, src, rec = _c2_case()
    nt = 4000
    m = make_model("psv", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    b = run_forward(m, nt, src, sid, rid, [0, 31], displacement=False)
    for q, s in enumerate((0, 31)):
        ref = _oracle_traces("f64", "psv", nx, nz, h, dt, nt, params, absorb, src, rec, s)
        for c in (0, 2):
            assert rel(traces(b, c)[q], ref["xyz"[c]]) < TRACE_TOL, (s, c)


def test_spin_nt2000_vs_fp64():
    """Micropolar spin (the tiled kernel) over 2000 steps, two shots, spin
    parameters in the ratios of the reference's spin example."""
    nx, nz, h, dt, nt = 160, 120, 2.0, 2e-4, 2000
    rng = np.random.default_rng(12)
    n = nx * nz
    base = dict(rho=2700.0, lam=8.1e9, mu=8.1e9, nu=10.05e8, j=2700.0, mu_c=1.5e8, nu_c=3.0e8)
    params = {k: (v * (1 + 0.05 * rng.uniform(-1, 1, n))).astype(np.float32) for k, v in base.items()}
    absorb = (20, 0.015, 1, 1, 1, 0)
    src = np.array([[60 * h, 40 * h, 0, 60.0, 0.02, 30.0, 1e10], [110 * h, 70 * h, 0, 55.0, 0.022, -45.0, 1e10]])
    rec = np.array([[(r + 0.5) * nx / 40 * h, 15 * h] for r in range(40)])
    m = make_model("spin", nx, nz, h, h, dt, params, absorb)
    sid = point_ids(src, np.float32(h), np.float32(h), nz)
    rid = point_ids(rec, np.float32(h), np.float32(h), nz)
    b = run_forward(m, nt, src, sid, rid, [0, 1])
    for s in range(2):
        ref = _oracle_traces("f64", "spin", nx, nz, h, dt, nt, params, absorb, src, rec, s)
        for c in (0, 2, 1):
            assert np.abs(ref["xyz"[c]]).max() > 0
            assert rel(traces(b, c)[s], ref["xyz"[c]]) < TRACE_TOL, (s, c)


def test_uneven_48_instances_full_length_vs_fp64():
    """The 48-instance uneven batch (grids 128-768, nt 1500-6000, 8-32
    shots), stepped as one CUDA-graph replay; eight instances, SH and
    P-SV, checked shot 0 against the FP64 oracle over their full nt."""
    from seispie_b200.uneven import UnevenBatch, make_instances
    from tests.gpu_helpers import oracle_trace_error
    insts = make_instances(48, seed=0)
    ub = UnevenBatch(insts)
    g = ub.capture()
    g.replay()
    torch.cuda.synchronize()
    picks = (0, 7, 13, 18, 25, 31, 36, 47)
    assert {insts[k].mode for k in picks} == {"sh", "psv"}
    for k in picks:
        assert oracle_trace_error(insts[k], ub.traces(k), insts[k].nt) < TRACE_TOL, k


def test_c2_exact_gradient_directional_fd():
    """The exact mu gradient at the full gradient configuration (512 x 512,
    32 shots, 256 receivers, nt 4000, checkpointed recomputation) against a
    central difference of the misfit along a smooth perturbation of mu."""
    from seispie_b200.adjoint import AcquisitionSetup, Seismograms, waveform_misfit
    from seispie_b200.engine import Grid
    nx, nz, h, dt, params, absorb, src, rec = _c2_case()
    nt = 4000
    setup = AcquisitionSetup("psv", Grid(nx, nz, h, h), dt, nt, src, rec, absorb)
    rho = torch.full((nx, nz), 2600.0, device="cuda")
    vp = torch.full((nx, nz), 3000.0, device="cuda")

    def lame(vs):
        return rho * (vp * vp - 2 * vs * vs), rho * vs * vs

    vs_true = torch.as_tensor(params["vs"].reshape(nx, nz), device="cuda")
    with torch.no_grad():
        lt, mt = lame(vs_true)
        data = Seismograms.apply(lt, mt, rho, setup).detach()
    lam, mu = lame(torch.full((nx, nz), 1732.0, device="cuda"))
    mu = mu.clone().requires_grad_(True)
    chi = waveform_misfit(Seismograms.apply(lam, mu, rho, setup), data, dt)
    chi.backward()
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    direction = torch.as_tensor((0.5 + 0.5 * np.sin(0.031 * i + 0.017 * j)) * 1732.0 ** 2 * 2600.0,
                                device="cuda", dtype=torch.float32)
    dd = float((mu.grad.double() * direction.double()).sum())
    eps = 1e-3
    with torch.no_grad():
        vals = [float(waveform_misfit(Seismograms.apply(lam, mu.detach() + sg * eps * direction, rho, setup),
                                      data, dt)) for sg in (1.0, -1.0)]
    fd = (vals[0] - vals[1]) / (2 * eps)
    assert abs(dd - fd) < 1e-3 * abs(fd), (dd, fd)
