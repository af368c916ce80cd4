"""CPU oracle for seispie's fd2d solver path -- TEST INFRASTRUCTURE ONLY.

This module is the checker for seispie_b200's CUDA path.  It is imported only
by tests/, by ``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg;
the product package never imports it and has no CPU fallback.

The stencil arithmetic lives in ``fd2d_oracle.c`` (built by ``oracle/Makefile``
into ``oracle/_build/liboracle_{f32,f64}.so``).  This file adds the host-side
pieces of the reference restated in numpy, and ctypes bindings:

* ``ricker``            seispie/solver/source/ricker.py:7-11
* ``grid_geometry``     seispie/solver/fd2d/fd2d.py:189-196
* ``point_ids``         seispie/solver/fd2d/fd2d.py:131-134, 156-159
* ``source_time_functions``  fd2d.py:127-138
* ``Oracle.forward / adjoint_sh / adjoint_psv / misfit / smooth``
                        solver.py:166-329, waveform.py:5-34, fd2d.py:76-108

Two precisions: ``"f32"`` repeats the reference's simulator arithmetic
(float32 everywhere, no FMA); ``"f64"`` is the FP64 oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIBS: dict[str, ctypes.CDLL] = {}

# model-parameter and state slot order shared with fd2d_oracle.c
PARAMS = ("rho", "lam", "mu", "bound", "nu", "j", "mu_c", "nu_c")
STATE = ("vx", "vz", "ux", "uz", "sxx", "szz", "sxz", "vy", "uy", "sxy", "szy",
         "vy_c", "uy_c", "syx_c", "syy_c", "syz_c")


def build() -> None:
    """Compile the oracle libraries (both precisions) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(prec: str) -> ctypes.CDLL:
    if prec not in ("f32", "f64"):
        raise ValueError("prec must be 'f32' or 'f64'")
    if prec not in _LIBS:
        path = os.path.join(_BUILD, "liboracle_%s.so" % prec)
        if not os.path.exists(path):
            build()
        _LIBS[prec] = ctypes.CDLL(path)
        _LIBS[prec].orc_misfit.restype = ctypes.c_double
    return _LIBS[prec]


def dtype_of(prec: str):
    return np.float32 if prec == "f32" else np.float64


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _ptr_table(arrays):
    tab = (ctypes.c_void_p * len(arrays))()
    for q, a in enumerate(arrays):
        tab[q] = None if a is None else a.ctypes.data
    return tab


# ----------------------------------------------------------------- host side

def ricker(t, f0, t0, ang, amp):
    """ricker.py:7-11, float64 numpy arithmetic, returns (x, y, z)."""
    a = (np.pi * f0) ** 2
    stf = -amp * (1.0 - 2.0 * a * (t - t0) ** 2) * np.exp(-a * (t - t0) ** 2)
    ang_rad = np.deg2rad(ang)
    return stf * np.sin(ang_rad), stf, -stf * np.cos(ang_rad)


def source_time_functions(src: np.ndarray, nt: int, dt: float):
    """fd2d.py:127-138: float32 stf_x/y/z of shape [nsrc*nt], one scalar
    ricker() call per sample as the reference loop does."""
    nsrc = src.shape[0]
    out = [np.zeros(nsrc * nt, dtype=np.float32) for _ in range(3)]
    for isrc in range(nsrc):
        for it in range(nt):
            x, y, z = ricker(it * dt, *src[isrc][3:])
            k = isrc * nt + it
            out[0][k], out[1][k], out[2][k] = x, y, z
    return out


def grid_geometry(x: np.ndarray, z: np.ndarray, npt):
    """fd2d.py:189-196.  x, z are float32 coordinate arrays, npt is np.int32.
    Returns (nx, nz, dx, dz) with dx, dz numpy float32 as in the reference."""
    lx = x.max() - x.min()
    lz = z.max() - z.min()
    nx = int(np.rint(np.sqrt(npt * lx / lz)))
    nz = int(np.rint(np.sqrt(npt * lz / lx)))
    return nx, nz, lx / (nx - 1), lz / (nz - 1)


def point_ids(points: np.ndarray, dx, dz, nz: int) -> np.ndarray:
    """fd2d.py:131-134 / 156-159: int(round-half-even(x/dx))*nz + ...(z/dz)."""
    ids = np.zeros(points.shape[0], dtype=np.int32)
    for q in range(points.shape[0]):
        px = int(np.round(points[q][0] / dx))
        pz = int(np.round(points[q][1] / dz))
        ids[q] = px * nz + pz
    return ids


# -------------------------------------------------------------- C restated

class Oracle:
    """Thin ctypes front end over fd2d_oracle.c in one precision."""

    def __init__(self, prec: str = "f64"):
        self.prec = prec
        self.dt = dtype_of(prec)
        self.lib = _lib(prec)

    def arr(self, a):
        return np.ascontiguousarray(a, dtype=self.dt)

    def vps2lm(self, vp, vs, rho):
        lam, mu, rho = self.arr(vp).copy(), self.arr(vs).copy(), self.arr(rho)
        self.lib.orc_vps2lm(_p(lam), _p(mu), _p(rho), ctypes.c_long(lam.size))
        return lam, mu

    def lm2vps(self, lam, mu, rho):
        vp, vs, rho = self.arr(lam).copy(), self.arr(mu).copy(), self.arr(rho)
        self.lib.orc_lm2vps(_p(vp), _p(vs), _p(rho), ctypes.c_long(vp.size))
        return vp, vs

    def set_bound(self, nx, nz, width, alpha, left, right, bottom, top):
        b = np.zeros(nx * nz, dtype=self.dt)
        self.lib.orc_set_bound(_p(b), nx, nz, int(width), ctypes.c_double(alpha),
                               int(left), int(right), int(bottom), int(top))
        return b

    def new_state(self, npt):
        return {name: np.zeros(npt, dtype=self.dt) for name in STATE}

    def forward(self, mode, nx, nz, dx, dz, dt, nt, params, src_id, stf, isrc, rec_id,
                sae=0, nsa=0, snapshots=False, state=None):
        """run_forward (solver.py:166-242).  mode in {'sh','psv','spin'}.
        ``params``: dict name->array (rho, lam, mu, bound [, nu, j, mu_c, nu_c]).
        ``stf``: (stf_x, stf_y, stf_z) each [nsrc*nt].  Returns (obs dict,
        state dict, snapshot dict)."""
        sh, psv, spin = mode == "sh", mode in ("psv", "spin"), mode == "spin"
        npt = nx * nz
        p = {k: self.arr(v) for k, v in params.items()}
        ptab = _ptr_table([p.get(k) for k in PARAMS])
        st = state if state is not None else self.new_state(npt)
        stab = _ptr_table([st[k] for k in STATE])
        nrec = len(rec_id)
        obs = {c: np.zeros(nrec * nt, dtype=self.dt) for c in "xyz"}
        src_id = np.ascontiguousarray(src_id, dtype=np.int32)
        rec_id = np.ascontiguousarray(rec_id, dtype=np.int32)
        stf = [self.arr(s) for s in stf]
        snaps = {}
        if snapshots and sae:
            for c in ("ux", "uz", "uy", "vx", "vz", "vy"):
                snaps[c] = np.zeros(nsa * npt, dtype=self.dt)
        g = snaps.get
        self.lib.orc_forward(int(sh), int(psv), int(spin), nx, nz, ctypes.c_double(dx), ctypes.c_double(dz),
                             ctypes.c_double(dt), nt, ptab, stab, len(src_id), _p(src_id),
                             _p(stf[0]), _p(stf[1]), _p(stf[2]), int(isrc), nrec, _p(rec_id),
                             _p(obs["x"]), _p(obs["y"]), _p(obs["z"]), int(sae), int(nsa),
                             _p(g("ux")), _p(g("uz")), _p(g("uy")), _p(g("vx")), _p(g("vz")), _p(g("vy")))
        return obs, st, {k: v.reshape(nsa, npt) for k, v in snaps.items()}

    def adjoint_sh(self, nx, nz, dx, dz, dt, nt, params, rec_id, adstf_y, sae, uy_fwd, k_mu, state=None):
        """run_adjoint SH branch (solver.py:290-321); accumulates into k_mu."""
        npt = nx * nz
        p = {k: self.arr(v) for k, v in params.items()}
        ptab = _ptr_table([p.get(k) for k in PARAMS])
        st = state if state is not None else self.new_state(npt)
        stab = _ptr_table([st[k] for k in STATE])
        rec_id = np.ascontiguousarray(rec_id, dtype=np.int32)
        adstf_y, uy_fwd = self.arr(adstf_y), self.arr(uy_fwd)
        assert k_mu.dtype == self.dt and k_mu.flags.c_contiguous
        self.lib.orc_adjoint_sh(nx, nz, ctypes.c_double(dx), ctypes.c_double(dz), ctypes.c_double(dt), nt,
                                ptab, stab, len(rec_id), _p(rec_id), _p(adstf_y), int(sae), _p(uy_fwd), _p(k_mu))
        return st

    def adjoint_psv(self, nx, nz, dx, dz, dt, nt, params, rec_id, adstf_x, adstf_z, sae,
                    snaps, k_lam, k_mu, k_rho, state=None):
        """P-SV adjoint as defined in fd2d_oracle.c (the reference's branch is
        broken); accumulates into k_lam, k_mu, k_rho."""
        npt = nx * nz
        p = {k: self.arr(v) for k, v in params.items()}
        ptab = _ptr_table([p.get(k) for k in PARAMS])
        st = state if state is not None else self.new_state(npt)
        stab = _ptr_table([st[k] for k in STATE])
        rec_id = np.ascontiguousarray(rec_id, dtype=np.int32)
        ax, az = self.arr(adstf_x), self.arr(adstf_z)
        sn = {k: self.arr(v) for k, v in snaps.items()}
        for k in (k_lam, k_mu, k_rho):
            assert k.dtype == self.dt and k.flags.c_contiguous
        self.lib.orc_adjoint_psv(nx, nz, ctypes.c_double(dx), ctypes.c_double(dz), ctypes.c_double(dt), nt,
                                 ptab, stab, len(rec_id), _p(rec_id), _p(ax), _p(az), int(sae),
                                 _p(sn["ux"]), _p(sn["uz"]), _p(sn.get("vx")), _p(sn.get("vz")),
                                 _p(k_lam), _p(k_mu), _p(k_rho))
        return st

    def misfit(self, data, syn, nt, dt, nrec):
        """waveform (waveform.py:5-34): returns (norm, adstf, residual)."""
        data, syn = self.arr(data), self.arr(syn)
        adstf = np.zeros(nrec * nt, dtype=self.dt)
        resid = np.zeros(nrec * nt, dtype=self.dt)
        norm = self.lib.orc_misfit(_p(data), _p(syn), _p(adstf), _p(resid), nt, ctypes.c_double(dt), nrec)
        return norm, adstf, resid

    def smooth(self, data, nx, nz, sigma):
        """smooth (fd2d.py:349-352) with init_gausian; returns a new array."""
        d = self.arr(data).copy()
        self.lib.orc_smooth(_p(d), nx, nz, int(sigma))
        return d
