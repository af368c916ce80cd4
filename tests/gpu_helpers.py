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
                chunks=None):
    """Forward for len(isrcs) shots (isrc -1 = all sources).  Returns the
    batch.  ``chunks`` splits the time loop into several fwi_run calls."""
    nsa = nt // sae if sae else 0
    b = ShotBatch(m, len(isrcs), nt, rec_id, sae=sae, nsa=nsa, snapshots=snapshots, snap_velocity=snap_velocity,
                  tile=tile)
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
