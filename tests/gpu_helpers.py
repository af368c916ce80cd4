"""Helpers that drive the CUDA path through the C-ABI for the GPU tests.

Everything here calls libseispie_b200.so through seispie_b200.engine; the
oracle is only used by the tests as the checker.
"""
from __future__ import annotations

import numpy as np
import torch

from seispie_b200 import _lib, engine
from seispie_b200._lib import FWI_PSV, FWI_SH, FWI_SPIN, check, ptr
from seispie_b200.engine import DeviceModel, Grid, ShotBatch

MODE = {"sh": FWI_SH, "psv": FWI_PSV, "spin": FWI_SPIN}


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make_model(mode, nx, nz, dx, dz, dt, params, absorb, device="cuda"):
    """params: rho + (vp, vs) or, for spin, lam, mu, nu, j, mu_c, nu_c.
    absorb: (width, alpha, left, right, bottom, top)."""
    return engine.build_model(mode, Grid(nx, nz, float(dx), float(dz)), dt, params, absorb, device)


def run_forward(m, nt, src, src_id, rec_id, isrcs, tile=0, sae=0, snapshots=False, snap_velocity=False,
                chunks=None, displacement=True):
    """Forward for len(isrcs) shots (isrc -1 = all sources).  Returns the
    batch.  ``chunks`` splits the time loop into several fwi_run calls;
    ``displacement`` False runs a displacement-free batch (row-marching
    kernel), True the tiled kernel variant ``tile``."""
    nsa = nt // sae if sae else 0
    b = ShotBatch(m, len(isrcs), nt, rec_id, sae=sae, nsa=nsa, snapshots=snapshots, snap_velocity=snap_velocity,
                  tile=tile, displacement=displacement)
    stf, _ = engine.ricker_stf(np.asarray(src, np.float64), nt, m.dt, m.device)
    inj = engine.injection_lists(len(isrcs), src_id, lambda s: isrcs[s])
    d = b.desc(inj=inj, stf=stf)
    b.clear()
    if chunks is None:
        b.run(d, False, 0, nt)
    else:
        it = 0
        for n in chunks:
            b.run(d, False, it, n)
            it += n
        assert it == nt
    b._stf = stf
    return b


def traces(b, comp):
    return b.traces(comp).cpu().numpy().reshape(b.nshots, -1)


def state(b, name):
    return b.field(name).cpu().numpy().reshape(b.nshots, -1)


def oracle_trace_error(inst, traces, nsteps: int, shot: int = 0) -> float:
    """Relative L2 error of one shot's first nsteps trace samples of an
    uneven-batch instance (seispie_b200.uneven.Instance) against the FP64
    oracle run for nsteps steps (host)."""
    from oracle.oracle import Oracle, point_ids as opids, source_time_functions
    o = Oracle("f64")
    lam, mu = o.vps2lm(inst.params["vp"], inst.params["vs"], inst.params["rho"])
    p = dict(rho=inst.params["rho"], lam=lam, mu=mu, bound=o.set_bound(inst.nx, inst.nz, *inst.absorb))
    h = np.float32(inst.h)
    sid = opids(inst.src, h, h, inst.nz)
    rid = opids(inst.rec, h, h, inst.nz)
    stf = source_time_functions(inst.src, nsteps, inst.dt)
    obs, _, _ = o.forward(inst.mode, inst.nx, inst.nz, float(h), float(h), inst.dt, nsteps, p, sid, stf, shot, rid)
    num = den = 0.0
    for c in range(3):
        if traces[c] is None:
            continue
        got = traces[c][shot, :, :nsteps].double().cpu().numpy().reshape(-1)
        ref = obs["xyz"[c]].reshape(len(rid), nsteps).reshape(-1)
        num += float(np.sum((got - ref) ** 2))
        den += float(np.sum(ref ** 2))
    return (num / den) ** 0.5 if den > 0 else 0.0
