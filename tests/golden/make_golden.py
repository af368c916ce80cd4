"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs icui/seispie's own ``seispie.solver.fd2d`` plugin, unchanged, under
Numba's CUDA simulator (NUMBA_ENABLE_CUDASIM=1), on grids small enough for the
simulator (about 1e3 cell-updates/s), and saves inputs and outputs as .npz.
The reference checkout is named by --reference (or the SEISPIE_REFERENCE
environment variable); it only has to exist when this script runs, never when
the tests run.

    python tests/golden/make_golden.py --reference PATH [--only NAME ...]

Each case drives the plugin exactly as sprun would (scripts/sprun:79-86):
``config`` is a dict of strings, ``path`` a dict of paths, ``mpi`` is None.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import time

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
REFERENCE = None  # set from --reference / SEISPIE_REFERENCE before any case runs

import numpy as np  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def write_model(d, nx, nz, dx, dz, fields):
    """Model files in the reference's format (fd2d.py:174-182)."""
    npt = np.array([nx * nz], dtype="int32")
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    allf = dict(fields)
    allf["x"] = (i * dx).ravel()
    allf["z"] = (j * dz).ravel()
    for k, v in allf.items():
        with open(os.path.join(d, "proc000000_%s.bin" % k), "wb") as f:
            npt.tofile(f)
            np.asarray(v, dtype="float32").ravel().tofile(f)


def smooth_field(rng, nx, nz, scale):
    """A smooth random perturbation (sum of a few low-order modes)."""
    x = np.linspace(0, 1, nx)[:, None]
    z = np.linspace(0, 1, nz)[None, :]
    f = np.zeros((nx, nz))
    for _ in range(4):
        a, b, c = rng.uniform(0.5, 3.0, 3)
        f += rng.uniform(-1, 1) * np.sin(np.pi * (a * x + b * z + c))
    return (scale * f / max(1e-12, np.abs(f).max())).ravel()


def base_config(**kw):
    cfg = dict(nt="30", dt="1e-3", sh="no", psv="no", spin="no", threads_per_block="64",
               abs_left="yes", abs_right="yes", abs_top="no", abs_bottom="yes",
               abs_width="5", abs_alpha="0.05", save_coordinates="", combine_sources="yes",
               save_snapshot="0", adjoint_interval="3", smooth="2")
    cfg.update({k: str(v) for k, v in kw.items()})
    return cfg


def make_solver(cfg, paths):
    from seispie.solver.fd2d import fd2d
    s = fd2d()
    s.config = cfg
    s.path = paths
    s.mpi = None
    s.setup(None)
    return s


def host(a):
    return a.copy_to_host()


def fwd_case(name, mode, nx, nz, h, nt, dt, src, rec, model, absorb, combine="yes", taskid=None):
    td = tempfile.mkdtemp()
    write_model(td, nx, nz, h, h, model)
    np.savetxt(td + "/src.dat", np.asarray(src, dtype=float))
    np.savetxt(td + "/rec.dat", np.asarray(rec, dtype=float))
    flags = dict(sh="yes" if mode == "sh" else "no", psv="yes" if mode in ("psv", "spin") else "no",
                 spin="yes" if mode == "spin" else "no")
    cfg = base_config(nt=nt, dt=dt, combine_sources=combine, **flags, **absorb)
    s = make_solver(cfg, dict(model_true=td, model_init=td, sources=td + "/src.dat",
                              stations=td + "/rec.dat", output=td))
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    if taskid is not None:
        s.taskid = taskid
    t0 = time.time()
    s.run_forward()
    el = time.time() - t0
    out = dict(mode=mode, nx=s.nx, nz=s.nz, dx=np.float32(s.dx), dz=np.float32(s.dz), dt=float(dt), nt=nt,
               src=np.asarray(src, dtype=float), rec=np.asarray(rec, dtype=float),
               src_id=host(s.src_id), rec_id=host(s.rec_id),
               stf_x=host(s.stf_x), stf_y=host(s.stf_y), stf_z=host(s.stf_z),
               rho=host(s.rho), lam=host(s.lam), mu=host(s.mu), bound=host(s.bound),
               isrc=-1 if combine == "yes" else taskid,
               config=np.array(repr(cfg)))
    for k, v in model.items():
        out["model_" + k] = np.asarray(v, dtype="float32")
    if mode == "spin":
        for k in ("nu", "j", "mu_c", "nu_c"):
            out[k] = host(getattr(s, k))
    fields = []
    if mode == "sh":
        fields = ["vy", "uy", "sxy", "szy"]
        out["obs_y"] = host(s.obs_y)
    else:
        fields = ["vx", "vz", "ux", "uz", "sxx", "szz", "sxz"]
        out["obs_x"] = host(s.obs_x)
        out["obs_z"] = host(s.obs_z)
        if mode == "spin":
            fields += ["vy_c", "uy_c", "syx_c", "syy_c", "syz_c"]
            out["obs_y"] = host(s.obs_y)
    for f in fields:
        out["state_" + f] = host(getattr(s, f))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print("%-16s %dx%d nt=%d  %.1fs" % (name, s.nx, s.nz, nt, el))


def case_sh_fwd():
    rng = np.random.default_rng(11)
    nx, nz, h = 20, 28, 10.0
    n = nx * nz
    model = dict(vp=3000 + smooth_field(rng, nx, nz, 150), vs=1732 + smooth_field(rng, nx, nz, 120),
                 rho=2600 + smooth_field(rng, nx, nz, 100))
    # receivers at exact half-cells check round-half-even (25/10 -> 2, 35/10 -> 4)
    src = [[95.0, 135.0, 0, 12.0, 0.09, 0.0, 1e10], [135.0, 175.0, 0, 9.0, 0.1, 0.0, -6e9]]
    rec = [[25.0, 35.0], [150.0, 40.0], [40.0, 205.0], [175.0, 255.0]]
    fwd_case("sh_fwd", "sh", nx, nz, h, 40, 1e-3, src, rec, model,
             dict(abs_left="yes", abs_right="yes", abs_top="no", abs_bottom="yes"))
    fwd_case("sh_fwd_task1", "sh", nx, nz, h, 24, 1e-3, src, rec, model,
             dict(abs_left="no", abs_right="yes", abs_top="yes", abs_bottom="no"), combine="no", taskid=1)


def case_psv_fwd():
    rng = np.random.default_rng(12)
    nx, nz, h = 24, 20, 10.0
    vp = 3000 + smooth_field(rng, nx, nz, 200)
    vs = 1732 + smooth_field(rng, nx, nz, 150)
    vp[:3] = 1000.0  # vp <= vs branch of vps2lm (lambda = 0)
    model = dict(vp=vp, vs=vs, rho=2600 + smooth_field(rng, nx, nz, 100))
    src = [[115.0, 95.0, 0, 10.0, 0.1, 30.0, 1e10], [75.0, 125.0, 0, 12.0, 0.08, 0.0, 5e9],
           [165.0, 55.0, 0, 8.0, 0.12, -70.0, 8e9]]
    rec = [[45.0, 45.0], [125.0, 25.0], [205.0, 165.0]]
    fwd_case("psv_fwd", "psv", nx, nz, h, 36, 1e-3, src, rec, model,
             dict(abs_left="yes", abs_right="no", abs_top="yes", abs_bottom="no"))


def case_spin_fwd():
    rng = np.random.default_rng(13)
    nx, nz, h = 20, 22, 2.0
    base = dict(rho=2700.0, **{"lambda": 8.1e9}, mu=8.1e9, nu=10.05e8, j=2700.0, lambda_c=7.75e8,
                mu_c=1.5e8, nu_c=3.0e8)
    model = {k: v * (1 + smooth_field(rng, nx, nz, 0.05)) for k, v in base.items()}
    src = [[19.0, 21.0, 0, 60.0, 0.02, 20.0, 1e10]]
    rec = [[9.0, 9.0], [29.0, 31.0]]
    fwd_case("spin_fwd", "spin", nx, nz, h, 30, 2e-4, src, rec, model,
             dict(abs_left="yes", abs_right="yes", abs_top="yes", abs_bottom="yes"))


def case_sh_grad():
    """The adjoint workflow (workflow/adjoint.py:14-30) at toy size, run as the
    steps of run_kernel(adj=1) (solver.py:332-404) so intermediates can be
    saved: traces from the true model, then forward/misfit/adjoint per shot
    on the initial model, then smoothing."""
    rng = np.random.default_rng(14)
    nx, nz, h = 16, 20, 10.0
    true = dict(vp=np.full(nx * nz, 3000.0), vs=1732 + smooth_field(rng, nx, nz, 200), rho=np.full(nx * nz, 2600.0))
    init = dict(vp=np.full(nx * nz, 3000.0), vs=np.full(nx * nz, 1732.0), rho=np.full(nx * nz, 2600.0))
    td_t, td_i, td_o = tempfile.mkdtemp(), tempfile.mkdtemp(), tempfile.mkdtemp()
    write_model(td_t, nx, nz, h, h, true)
    write_model(td_i, nx, nz, h, h, init)
    src = [[55.0, 45.0, 0, 14.0, 0.07, 0.0, 1e10], [105.0, 45.0, 0, 14.0, 0.07, 0.0, 1e10]]
    rec = [[35.0, 145.0], [75.0, 145.0], [115.0, 145.0]]
    np.savetxt(td_o + "/src.dat", np.asarray(src))
    np.savetxt(td_o + "/rec.dat", np.asarray(rec))
    nt, sae, sigma = 30, 3, 2
    cfg = base_config(nt=nt, dt=1e-3, sh="yes", combine_sources="no", adjoint_interval=sae, smooth=sigma)
    s = make_solver(cfg, dict(model_true=td_t, model_init=td_i, sources=td_o + "/src.dat",
                              stations=td_o + "/rec.dat", output=td_o))
    t0 = time.time()
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.import_traces()
    data = [d.copy() for d in s.syn_y]
    s.import_model(0)
    s.setup_adjoint()
    s.clear_kernels()
    misfit = 0
    adstf = []
    for i in range(s.nsrc):
        s.taskid = i
        s.run_forward()
        misfit += s._compute_misfit("y", s.syn_y[i])
        adstf.append(host(s.adstf_y))
        s.run_adjoint()
    k_raw = host(s.k_mu)
    s.smooth(s.k_mu)
    k_smooth = host(s.k_mu)
    np.savez_compressed(os.path.join(OUT, "sh_grad.npz"), nx=s.nx, nz=s.nz, dx=np.float32(s.dx), dz=np.float32(s.dz),
                        dt=1e-3, nt=nt, sae=sae, sigma=sigma, src=np.asarray(src), rec=np.asarray(rec),
                        src_id=host(s.src_id), rec_id=host(s.rec_id), stf_y=host(s.stf_y),
                        true_vs=true["vs"].astype("float32"), rho=host(s.rho), mu=host(s.mu), lam=host(s.lam),
                        bound=host(s.bound), data=np.stack(data), adstf=np.stack(adstf),
                        misfit=np.float64(misfit), k_mu_raw=k_raw, k_mu=k_smooth, config=np.array(repr(cfg)))
    print("%-16s %dx%d nt=%d  %.1fs  misfit=%g" % ("sh_grad", nx, nz, nt, time.time() - t0, misfit))


def case_misfit_smooth():
    from seispie.solver.misfit.waveform import waveform
    from numba import cuda
    rng = np.random.default_rng(15)
    nt, nrec, dt = 50, 3, 2e-3
    data = rng.standard_normal(nt * nrec).astype("float32")
    syn = rng.standard_normal(nt * nrec).astype("float32")
    stream = cuda.stream()
    adstf = cuda.to_device(np.zeros(nt * nrec, dtype="float32"), stream=stream)
    norm = waveform(cuda.to_device(data), cuda.to_device(syn), adstf, nt, dt, nrec, stream)
    # smoothing through the plugin's own setup_adjoint/smooth
    nx, nz, sigma = 18, 24, 3
    td = tempfile.mkdtemp()
    write_model(td, nx, nz, 5.0, 5.0, dict(vp=np.full(nx * nz, 3000.0), vs=np.full(nx * nz, 1700.0),
                                            rho=np.full(nx * nz, 2500.0)))
    np.savetxt(td + "/src.dat", np.asarray([[20.0, 20.0, 0, 10.0, 0.1, 0.0, 1.0]]))
    np.savetxt(td + "/rec.dat", np.asarray([[30.0, 30.0]]))
    s = make_solver(base_config(nt=4, sh="yes", smooth=sigma), dict(model_true=td, model_init=td,
                    sources=td + "/src.dat", stations=td + "/rec.dat", output=td))
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    s.setup_adjoint()
    raw = (rng.standard_normal(nx * nz) * 1e-3).astype("float32")
    raw[nx * nz // 2] = 1.0
    d = cuda.to_device(raw)
    s.smooth(d)
    np.savez_compressed(os.path.join(OUT, "misfit_smooth.npz"), nt=nt, nrec=nrec, dt=dt, data=data, syn=syn,
                        misfit=np.float64(norm), adstf=adstf.copy_to_host(), nx=nx, nz=nz, sigma=sigma,
                        smooth_in=raw, smooth_out=d.copy_to_host(), gsum=host(s.gsum))
    print("%-16s misfit=%g" % ("misfit_smooth", norm))


def case_example_geometry():
    """Geometry of the reference's own examples/forward set-up (201x201,
    12 sources, 132 stations): nx/nz/dx/dz, src_id, rec_id and the first two
    source-time functions, through import_model/import_sources/import_stations."""
    ex = os.path.join(REFERENCE, "examples", "forward")
    cfg = base_config(nt=4800, dt=0.06, sh="yes", abs_width=20, abs_alpha=0.015,
                      abs_top="no", abs_bottom="yes", abs_left="yes", abs_right="yes")
    td = tempfile.mkdtemp()
    s = make_solver(cfg, dict(model_true=ex + "/model_true", model_init=ex + "/model_init",
                              sources=ex + "/sources.dat", stations=ex + "/stations.dat", output=td))
    t0 = time.time()
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    bound = host(s.bound)
    np.savez_compressed(os.path.join(OUT, "example_geometry.npz"), nx=s.nx, nz=s.nz, dx=np.float32(s.dx),
                        dz=np.float32(s.dz), npt=int(s.npt[0]), src=np.loadtxt(ex + "/sources.dat", ndmin=2),
                        rec=np.loadtxt(ex + "/stations.dat", ndmin=2), src_id=host(s.src_id),
                        rec_id=host(s.rec_id), stf_y01=host(s.stf_y)[: 2 * 4800], nt=4800, dt=0.06,
                        bound=bound, lam=host(s.lam), mu=host(s.mu))
    print("%-16s %dx%d  %.1fs" % ("example_geometry", s.nx, s.nz, time.time() - t0))


def case_optimize():
    """The reference's L-BFGS (with its backtracking line search) and CG
    (with the bracketing line search) on a weighted quadratic misfit, driven
    by the loop of optimize/base.py:28-50 with a stand-in solver; records every
    gradient, direction, line-search status and trial model."""
    from seispie.optimize.cg import cg
    from seispie.optimize.lbfgs import lbfgs
    rng = np.random.default_rng(16)
    n = 96
    w = rng.uniform(0.5, 4.0, n)
    mt = rng.uniform(2.0, 3.0, n)
    m0 = (mt + rng.uniform(-0.4, 0.4, n)).astype("float32")

    class Solver:
        def __init__(self):
            self.m = m0.copy()
            self.trials = []

        def update_model(self, m):
            self.m = np.asarray(m, dtype="float32").copy()
            self.trials.append(self.m.copy())

        def compute_misfit(self):
            return float(np.sum(w * (self.m.astype("float64") - mt) ** 2))

        def gradient(self):
            return (2 * w * (self.m.astype("float64") - mt)).astype("float32")

    class Workflow:
        pass

    out = dict(w=w, mt=mt, m0=m0)
    for name, cls in (("lbfgs", lbfgs), ("cg", cg)):
        s = Solver()
        wf = Workflow()
        wf.solver = s
        opt = cls()
        opt.config = dict(niter="6", ls_step="10", ls_step_max="0.5", ls_step_init="0.05", ls_thresh="1.2",
                          lbfgs_mem="3")
        opt.mpi = None
        opt.setup(wf)
        gs, ps, st, ms, mis, ntr = [], [], [], [], [], []
        for i in range(6):
            opt.g_new, misfit, opt.m_new = s.gradient(), s.compute_misfit(), s.m.copy()
            opt.p_new = opt.compute_direction()
            opt.m_old, opt.p_old, opt.g_old = opt.m_new, opt.p_new, opt.g_new
            status = opt.line_search(misfit)
            gs.append(opt.g_new)
            ps.append(np.asarray(opt.p_new, dtype="float32"))
            st.append(status)
            ms.append(s.m.copy())
            mis.append(misfit)
            ntr.append(len(s.trials))
            if status < 0:
                break
        out.update({name + "_g": np.stack(gs), name + "_p": np.stack(ps), name + "_status": np.array(st),
                    name + "_m": np.stack(ms), name + "_misfit": np.array(mis), name + "_ntrials": np.array(ntr)})
    np.savez_compressed(os.path.join(OUT, "optimize.npz"), **out)
    print("%-16s lbfgs status %s, cg status %s" % ("optimize", out["lbfgs_status"], out["cg_status"]))


CASES = dict(optimize=case_optimize, sh_fwd=case_sh_fwd, psv_fwd=case_psv_fwd, spin_fwd=case_spin_fwd, sh_grad=case_sh_grad,
             misfit_smooth=case_misfit_smooth, example_geometry=case_example_geometry)

if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SEISPIE_REFERENCE"),
                    help="root of the seispie checkout to run (the directory holding the seispie package)")
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    if not args.reference or not os.path.isdir(os.path.join(args.reference, "seispie")):
        ap.error("--reference (or SEISPIE_REFERENCE) must name the seispie checkout")
    REFERENCE = os.path.abspath(args.reference)
    sys.path.insert(0, REFERENCE)
    for name, fn in CASES.items():
        if args.only is None or name in args.only:
            fn()
