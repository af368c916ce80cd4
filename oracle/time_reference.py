"""Time the unmodified reference solver on this machine's CPU and record it.

Runs icui/seispie's own ``seispie.solver.fd2d`` plugin, unchanged, under
Numba's CUDA simulator (NUMBA_ENABLE_CUDASIM=1) -- the only way the
reference's solver runs without a GPU -- on the reduced grid its speed
allows (64 x 64; the simulator manages about 1e3 cell-updates/s, so the
512 x 512 x 32-shot gradient would take years), and writes
oracle/reference_cudasim.json with the cell-update rates.  bench.py reports
that record beside its own CPU baseline; it is test infrastructure, not
part of the package.

    python oracle/time_reference.py --reference PATH [--nt 20]

Cases: P-SV forward of one shot (run_forward, solver.py:166-287) and the SH
gradient of one shot (forward, misfit, adjoint with interaction; the
reference's P-SV adjoint cannot run, solver.py:324-329).  The simulator
serialises every thread under the GIL, so it uses one core whatever the
machine has; nproc is recorded beside the rates.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import tempfile
import time

import numpy as np

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cudasim.json")


def write_model(d, nx, nz, h, fields):
    """Model files in the reference's format: [int32 npt][float32 x npt]."""
    os.makedirs(d, exist_ok=True)
    npt = np.array([nx * nz], dtype="int32")
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    allf = dict(fields, x=(i * h).ravel(), z=(j * h).ravel())
    for k, v in allf.items():
        with open(os.path.join(d, "proc000000_%s.bin" % k), "wb") as f:
            npt.tofile(f)
            np.asarray(v, dtype="float32").ravel().tofile(f)


def solver(mode, nx, nt, td):
    from seispie.solver.fd2d import fd2d
    h = 10.0
    n = nx * nx
    write_model(td + "/true", nx, nx, h, dict(vp=np.full(n, 3000.0), vs=np.full(n, 1732.0) * 1.02,
                                              rho=np.full(n, 2600.0)))
    write_model(td + "/init", nx, nx, h, dict(vp=np.full(n, 3000.0), vs=np.full(n, 1732.0), rho=np.full(n, 2600.0)))
    np.savetxt(td + "/src.dat", np.array([[nx / 2 * h, 8 * h, 0, 10.0, 0.1, 0.0, 1e10]]))
    np.savetxt(td + "/rec.dat", np.array([[(r + 0.5) * nx / 8 * h, 10 * h] for r in range(8)]))
    os.makedirs(td + "/out", exist_ok=True)
    s = fd2d()
    s.config = dict(nt=str(nt), dt="1e-3", sh="yes" if mode == "sh" else "no", psv="yes" if mode == "psv" else "no",
                    spin="no", threads_per_block="64", abs_left="yes", abs_right="yes", abs_top="no",
                    abs_bottom="yes", abs_width="8", abs_alpha="0.015", save_coordinates="", combine_sources="no",
                    save_snapshot="0", adjoint_interval="5", smooth="2")
    s.path = dict(model_true=td + "/true", model_init=td + "/init", sources=td + "/src.dat",
                  stations=td + "/rec.dat", output=td + "/out")
    s.mpi = None
    s.setup(None)
    s.import_model(1)
    s.import_sources()
    s.import_stations()
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SEISPIE_REFERENCE"),
                    help="root of the seispie checkout (the directory holding the seispie package)")
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--nt", type=int, default=20)
    a = ap.parse_args()
    if not a.reference or not os.path.isdir(os.path.join(a.reference, "seispie")):
        ap.error("--reference (or SEISPIE_REFERENCE) must name the seispie checkout")
    sys.path.insert(0, os.path.abspath(a.reference))
    import numba
    rec = {"what": "unmodified seispie fd2d under NUMBA_ENABLE_CUDASIM=1, one shot, %dx%d, nt %d" % (a.nx, a.nx, a.nt),
           "numba": numba.__version__, "numpy": np.__version__, "python": platform.python_version(),
           "nproc": os.cpu_count(), "cores_used": 1, "machine": platform.machine(), "cases": {}}
    with tempfile.TemporaryDirectory() as td:
        s = solver("psv", a.nx, a.nt, td + "/psv")
        s.taskid = 0
        t = time.perf_counter()
        s.run_forward()
        el = time.perf_counter() - t
        rec["cases"]["psv_forward"] = dict(seconds=el, cell_updates=a.nx * a.nx * a.nt,
                                           cell_updates_per_s=a.nx * a.nx * a.nt / el)
        s = solver("sh", a.nx, a.nt, td + "/sh")
        s.import_traces()
        s.import_model(0)
        t = time.perf_counter()
        s.compute_gradient()
        el = time.perf_counter() - t
        # forward and adjoint counted separately, as the GPU bench counts them
        rec["cases"]["sh_gradient"] = dict(seconds=el, cell_updates=2 * a.nx * a.nx * a.nt,
                                           cell_updates_per_s=2 * a.nx * a.nx * a.nt / el)
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
