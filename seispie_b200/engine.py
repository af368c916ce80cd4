"""Device-side state of the solver: grids, models and shot batches.

PyTorch is used only to own device memory and streams; every computation is a
call into libseispie_b200.so.  Layout in HBM: a field of one shot is ``nx``
rows of ``pitch`` float32 (z contiguous, pitch = nz rounded up to 4 so that
16-byte staging copies stay aligned); the shots of a batch follow each other.
The model is shared by the shots of a batch.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import FWI_PSV, FWI_SH, FWI_SPIN, FwiBatch, check, ptr

NS = {FWI_SH: 2, FWI_PSV: 3, FWI_SPIN: 6}  # stress fields
NV = {FWI_SH: 1, FWI_PSV: 2, FWI_SPIN: 3}  # velocity / displacement components
# user-facing component slot (x=0, y=1, z=2) of each velocity component
COMP = {FWI_SH: (1,), FWI_PSV: (0, 2), FWI_SPIN: (0, 2, 1)}


def pitch_for(nz: int) -> int:
    return (nz + 3) // 4 * 4


def stream_handle(stream: torch.cuda.Stream | None) -> int | None:
    """cudaStream_t of ``stream``, or of torch's current stream when None, so
    that library calls are ordered with the torch copies around them."""
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream or None


@dataclass
class Grid:
    nx: int
    nz: int
    dx: float
    dz: float

    @property
    def pitch(self) -> int:
        return pitch_for(self.nz)

    @property
    def npt(self) -> int:
        return self.nx * self.nz


class DeviceModel:
    """Model parameters on the device in padded layout, plus the derived
    arrays of the step kernel (dt/rho, dt/j, mu_c+nu_c)."""

    def __init__(self, grid: Grid, mode: int, dt: float, device, stream=None):
        self.grid, self.mode, self.dt, self.device, self.stream = grid, mode, float(dt), device, stream
        shape = (grid.nx, grid.pitch)
        names = ["rho", "lam", "mu", "bound", "buo"]
        if mode == FWI_SPIN:
            names += ["nu", "j", "mu_c", "nu_c", "buo_j", "mnc"]
        with torch.cuda.stream(stream) if stream is not None else _null():
            for n in names:
                setattr(self, n, torch.zeros(shape, dtype=torch.float32, device=device))

    def pad(self, host: np.ndarray) -> torch.Tensor:
        """Upload a reference-layout [npt] float32 array into padded layout."""
        g = self.grid
        t = torch.zeros((g.nx, g.pitch), dtype=torch.float32, device=self.device)
        src = torch.from_numpy(np.ascontiguousarray(host, dtype=np.float32).reshape(g.nx, g.nz))
        with torch.cuda.stream(self.stream) if self.stream is not None else _null():
            t[:, : g.nz].copy_(src.pin_memory() if torch.cuda.is_available() else src, non_blocking=True)
        return t

    def set(self, name: str, host: np.ndarray) -> None:
        getattr(self, name).copy_(self.pad(host))

    def unpad(self, t: torch.Tensor) -> torch.Tensor:
        return t[:, : self.grid.nz].reshape(-1)

    def prepare(self) -> None:
        g = self.grid
        n = g.nx * g.pitch
        s = stream_handle(self.stream)
        if self.mode == FWI_SPIN:
            check(_lib.load().fwi_prepare_model(ptr(self.rho), ptr(self.j), ptr(self.mu_c), ptr(self.nu_c),
                                                self.dt, n, ptr(self.buo), ptr(self.buo_j), ptr(self.mnc), s),
                  "fwi_prepare_model")
        else:
            check(_lib.load().fwi_prepare_model(ptr(self.rho), None, None, None, self.dt, n, ptr(self.buo),
                                                None, None, s), "fwi_prepare_model")


class _null:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


def build_model(mode: str, grid: Grid, dt: float, params: dict, absorb, device="cuda", stream=None) -> DeviceModel:
    """A ready DeviceModel from host arrays in the reference's cell order.

    params: rho plus vp/vs (converted on the device by fwi_vps2lm, as
    import_model does, fd2d.py:214-216) or lam/mu; spin also needs nu, j,
    mu_c, nu_c.  absorb: (width, alpha, left, right, bottom, top) for
    fwi_set_bound (fd2d.py:220-228)."""
    m = DeviceModel(grid, _lib.MODES[mode], dt, device, stream)
    lib = _lib.load()
    s = stream_handle(stream)
    m.set("rho", params["rho"])
    if mode == "spin":
        for k in ("lam", "mu", "nu", "j", "mu_c", "nu_c"):
            m.set(k, params[k])
    elif "vp" in params:
        m.set("lam", params["vp"])
        m.set("mu", params["vs"])
        check(lib.fwi_vps2lm(ptr(m.lam), ptr(m.mu), ptr(m.rho), m.lam.numel(), s), "fwi_vps2lm")
    else:
        m.set("lam", params["lam"])
        m.set("mu", params["mu"])
    w, a, l, r, b, t = absorb
    check(lib.fwi_set_bound(ptr(m.bound), grid.nx, grid.nz, grid.pitch, int(w), float(a), int(l), int(r), int(b),
                            int(t), s), "fwi_set_bound")
    m.prepare()
    return m


def point_ids(points: np.ndarray, dx, dz, nz: int) -> np.ndarray:
    """Cell numbers of sources / stations (fd2d.py:131-134, 156-159):
    int(round-half-even(x/dx)) * nz + int(round-half-even(z/dz)), with the
    division in float64 by the float32 spacing, as numpy does."""
    ids = np.zeros(points.shape[0], dtype="int32")
    for q in range(points.shape[0]):
        px = int(np.round(points[q][0] / dx))
        pz = int(np.round(points[q][1] / dz))
        ids[q] = px * nz + pz
    return ids


# widest grid (z cells) the row-marching step kernel of displacement-free batches takes
MARCH_MAX_NZ = 1024


def displacement_free_ok(mode: int, grid: Grid, snapshots: bool = False) -> bool:
    """Whether a forward batch can run without displacement fields (the
    row-marching step kernel): SH or P-SV, nz <= 1024, no snapshots."""
    return mode in (FWI_SH, FWI_PSV) and grid.nz <= MARCH_MAX_NZ and not snapshots


class ShotBatch:
    """State of ``nshots`` concurrent shots on one model: ping-pong stress and
    velocity pairs, displacement, receiver traces and (optionally) the
    forward snapshots the adjoint needs.

    ``inj``: (ptr[nshots+1], cell[], row[]) int32 host arrays; entry e of shot
    s adds stf[row[e]*nt + it] at cell[e] (reference cell numbering).

    ``displacement``: keep displacement fields (True), or not (False: the
    traces are rebuilt from the velocity at the receivers, bit-identically,
    and the step runs on the row-marching kernel); None picks False wherever
    that kernel applies (``displacement_free_ok``).  ``tile`` selects the
    tiled kernel variant of batches with displacement fields.
    """

    def __init__(self, model: DeviceModel, nshots: int, nt: int, rec_cell: np.ndarray, sae: int = 0,
                 nsa: int = 0, snapshots: bool = False, snap_velocity: bool = False, tile: int = 0,
                 displacement: bool | None = None):
        self.model, self.grid, self.mode = model, model.grid, model.mode
        self.nshots, self.nt, self.sae, self.nsa = int(nshots), int(nt), int(sae), int(nsa)
        self.device, self.stream = model.device, model.stream
        g = self.grid
        if displacement is None:
            displacement = not displacement_free_ok(self.mode, g, snapshots)
        elif not displacement and not displacement_free_ok(self.mode, g, snapshots):
            raise ValueError("a displacement-free batch needs SH or P-SV, nz <= %d and no snapshots" % MARCH_MAX_NZ)
        self.has_disp = bool(displacement)
        shape = (self.nshots, g.nx, g.pitch)
        ns, nv = NS[self.mode], NV[self.mode]
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=self.device)  # noqa: E731
        with torch.cuda.stream(self.stream) if self.stream is not None else _null():
            self.sig = [[z(*shape) for _ in range(ns)] for _ in range(2)]
            self.vel = [[z(*shape) for _ in range(nv)] for _ in range(2)]
            self.disp = [z(*shape) for _ in range(nv)] if self.has_disp else []
            self.nrec = len(rec_cell)
            rc = np.asarray(rec_cell, dtype=np.int32)
            self.rec_cell = torch.as_tensor(rc).to(self.device)
            # receivers by cell (stable), for the row-marching kernel's walk
            self.rec_order = torch.as_tensor(np.argsort(rc, kind="stable").astype(np.int32)).to(self.device)
            self.obs = [None, None, None]
            for q in range(nv):
                self.obs[COMP[self.mode][q]] = z(self.nshots * max(self.nrec, 1) * self.nt)
            self.snap_u = [None, None, None]
            self.snap_v = [None, None, None]
            if snapshots:
                if sae < 1 or nsa < 1:
                    raise ValueError("snapshots need adjoint_interval >= 1 and nt >= adjoint_interval")
                for q in range(min(nv, 2)):
                    c = COMP[self.mode][q]
                    self.snap_u[c] = z(nsa, *shape)
                    if snap_velocity:
                        self.snap_v[c] = z(nsa, *shape)
        self.cur = 0
        self.tile = int(tile)
        self.ring = 0  # staging-ring depth of the row-marching kernel (0 = automatic)
        self.ctas_per_sm = 0  # row-marching grid: resident CTAs per SM (0 = all that fit)
        self.adj_tile = 0  # P-SV transposed step: 0 = 32 x 64 tiles, 1 = 32 x 32 tiles
        # programmatic dependent launch between the steps of one call (fwi_batch.step_overlap)
        self.step_overlap = 1

    # ------------------------------------------------------------ descriptors
    def desc(self, inj=None, stf=(None, None, None), record=True, kernels=(None, None, None)) -> FwiBatch:
        """kernels: FP64 accumulators (k_lam, k_mu, k_rho[, k_nu, k_mnc, k_buoj])."""
        g, m = self.grid, self.model
        b = FwiBatch()
        b.mode, b.nx, b.nz, b.pitch = self.mode, g.nx, g.nz, g.pitch
        b.nshots, b.nt, b.dx, b.dz, b.dt = self.nshots, self.nt, float(g.dx), float(g.dz), float(m.dt)
        b.cur, b.tile, b.ring, b.ctas_per_sm = self.cur, self.tile, self.ring, self.ctas_per_sm
        b.adj_tile = self.adj_tile
        b.step_overlap = self.step_overlap
        for h in range(2):
            for f, t in enumerate(self.sig[h]):
                b.sig[h][f] = ptr(t)
            for q, t in enumerate(self.vel[h]):
                b.vel[h][q] = ptr(t)
        for q, t in enumerate(self.disp):
            b.disp[q] = ptr(t)
        b.buo, b.bound, b.mu = ptr(m.buo), ptr(m.bound), ptr(m.mu)
        b.lam = ptr(m.lam)
        if self.mode == FWI_SPIN:
            b.buo_j, b.nu, b.mnc = ptr(m.buo_j), ptr(m.nu), ptr(m.mnc)
        if inj is not None:
            ip, ic, ir = upload_lists(inj, self.device)
            b._keep = [ip, ic, ir]
            b.inj_ptr, b.inj_cell, b.inj_row = ptr(ip), ptr(ic), ptr(ir)
            for c in range(3):
                b.stf[c] = ptr(stf[c])
        b.nrec = self.nrec
        b.rec_cell = ptr(self.rec_cell) if self.nrec else None
        b.rec_order = ptr(self.rec_order) if self.nrec else None
        for c in range(3):
            b.obs[c] = ptr(self.obs[c]) if record else None
            b.snap_u[c] = ptr(self.snap_u[c])
            b.snap_v[c] = ptr(self.snap_v[c])
        b.sae, b.nsa = self.sae, self.nsa
        kernels = tuple(kernels) + (None,) * (6 - len(kernels))
        b.k_lam, b.k_mu, b.k_rho, b.k_nu, b.k_mnc, b.k_buoj = (ptr(k) for k in kernels)
        return b

    def set_segment(self, b: FwiBatch, seg_e, seg_ds, seg0: int, nseg: int) -> FwiBatch:
        """Point a descriptor at per-step segment stores (exact adjoint):
        strain fields seg_e[k] and divergence per component slot seg_ds[c]."""
        for k in range(6):
            b.seg_e[k] = ptr(seg_e[k]) if k < len(seg_e) else None
        for c in range(3):
            b.seg_ds[c] = ptr(seg_ds[c])
        b.seg0, b.nseg = int(seg0), int(nseg)
        return b

    def run_transposed(self, desc: FwiBatch, it_hi: int, nsteps: int) -> None:
        desc.cur = self.cur
        check(_lib.load().fwi_run_transposed(ctypes.byref(desc), int(it_hi), int(nsteps),
                                             stream_handle(self.stream)), "fwi_run_transposed")
        self.cur = desc.cur

    def state_tensors(self):
        """Current wavefield tensors (stress, velocity, displacement)."""
        return self.sig[self.cur] + self.vel[self.cur] + self.disp

    def clear(self) -> None:
        """Zero the wavefields (clear_wavefields, fd2d.py:318-341)."""
        with torch.cuda.stream(self.stream) if self.stream is not None else _null():
            for h in range(2):
                for t in self.sig[h] + self.vel[h]:
                    t.zero_()
            for t in self.disp:
                t.zero_()
        self.cur = 0

    def run(self, desc: FwiBatch, adjoint: bool, it0: int, nsteps: int) -> None:
        desc.cur = self.cur
        check(_lib.load().fwi_run(ctypes.byref(desc), int(adjoint), int(it0), int(nsteps),
                                  stream_handle(self.stream)), "fwi_run")
        self.cur = desc.cur

    # ------------------------------------------------------------- accessors
    def field(self, name: str) -> torch.Tensor:
        """Current state field by the reference's name, [nshots, nx, nz]."""
        ns_names = {FWI_SH: ["sxy", "szy"], FWI_PSV: ["sxx", "szz", "sxz"],
                    FWI_SPIN: ["sxx", "szz", "sxz", "syx_c", "syy_c", "syz_c"]}[self.mode]
        v_names = {FWI_SH: ["vy"], FWI_PSV: ["vx", "vz"], FWI_SPIN: ["vx", "vz", "vy_c"]}[self.mode]
        u_names = {FWI_SH: ["uy"], FWI_PSV: ["ux", "uz"], FWI_SPIN: ["ux", "uz", "uy_c"]}[self.mode]
        nz = self.grid.nz
        if name in ns_names:
            return self.sig[self.cur][ns_names.index(name)][:, :, :nz]
        if name in v_names:
            return self.vel[self.cur][v_names.index(name)][:, :, :nz]
        if name in u_names:
            if not self.has_disp:
                raise KeyError("%s: this batch keeps no displacement fields (displacement=False)" % name)
            return self.disp[u_names.index(name)][:, :, :nz]
        raise KeyError(name)

    def traces(self, comp: int) -> torch.Tensor:
        """Receiver traces of component comp (0 x, 1 y, 2 z), [nshots, nrec, nt]."""
        return self.obs[comp].view(self.nshots, max(self.nrec, 1), self.nt)[:, : self.nrec]


def _sort_by_cell(ptr_: np.ndarray, cell: np.ndarray, row: np.ndarray) -> tuple:
    """Entries of every shot ordered by cell, stably: entries at one cell
    keep their order, so each cell's sum (taken in entry order) is
    unchanged; the row-marching step kernel visits them in this order."""
    for s in range(len(ptr_) - 1):
        lo, hi = int(ptr_[s]), int(ptr_[s + 1])
        o = np.argsort(cell[lo:hi], kind="stable")
        cell[lo:hi] = cell[lo:hi][o]
        row[lo:hi] = row[lo:hi][o]
    return ptr_, cell, row


def injection_lists(nshots: int, src_id: np.ndarray, isrc_of_shot) -> tuple:
    """CSR injection lists for a forward batch.  isrc_of_shot(s) returns -1
    for 'all sources' (combine_sources = yes) or the one source index of shot
    s (solver.py:180-183, stf_dsy's isrc test at solver.py:81).  The entries
    of a shot are ordered by cell, sources on one cell in source order."""
    ptr_, cell, row = [0], [], []
    for s in range(nshots):
        isrc = isrc_of_shot(s)
        idx = range(len(src_id)) if isrc < 0 else [isrc]
        for i in idx:
            cell.append(int(src_id[i]))
            row.append(int(i))
        ptr_.append(len(cell))
    return _sort_by_cell(np.asarray(ptr_, np.int32), np.asarray(cell, np.int32), np.asarray(row, np.int32))


def upload_lists(inj, device) -> tuple:
    """Injection lists (ptr, cell, row) as int32 device tensors; lists that
    are device tensors already are passed through (no host copy, so a
    descriptor built from them can be made during CUDA-graph capture)."""
    return tuple(a if isinstance(a, torch.Tensor) and a.is_cuda else
                 torch.as_tensor(np.asarray(a, dtype=np.int32)).to(device) for a in inj)


def adjoint_injection_lists(nshots: int, rec_id: np.ndarray) -> tuple:
    """Adjoint sources: every receiver of every shot, row = shot*nrec + r
    (solver.py:311: stf_dsy over rec_id with isrc = -1), ordered by cell
    within a shot (receivers on one cell in receiver order)."""
    nrec = len(rec_id)
    ptr_ = np.arange(nshots + 1, dtype=np.int32) * nrec
    cell = np.tile(np.asarray(rec_id, np.int32), nshots)
    row = np.arange(nshots * nrec, dtype=np.int32)
    return _sort_by_cell(ptr_, cell, row)


def ricker_stf(src: np.ndarray, nt: int, dt: float, device, stream=None):
    """stf_x, stf_y, stf_z [nsrc*nt] on the device (fwi_ricker)."""
    nsrc = src.shape[0]
    par = torch.as_tensor(np.ascontiguousarray(src[:, 3:7], dtype=np.float64)).to(device)
    out = [torch.zeros(nsrc * nt, dtype=torch.float32, device=device) for _ in range(3)]
    check(_lib.load().fwi_ricker(ptr(par), nsrc, nt, float(dt), ptr(out[0]), ptr(out[1]), ptr(out[2]),
                                 stream_handle(stream)), "fwi_ricker")
    return out, par


def check_device(stream=None, what: str = "") -> None:
    """Wait for ``stream`` (torch's current stream when None), then read and
    clear the library's device status: if a bounded wait in one of its
    kernels gave up (a copy that never landed), the results written since
    the last check are invalid, and this raises FwiError."""
    s = torch.cuda.current_stream() if stream is None else stream
    s.synchronize()
    v = ctypes.c_int()
    check(_lib.load().fwi_device_status(ctypes.byref(v), 1), "fwi_device_status")
    if v.value:
        kinds = [k for bit, k in ((1, "step"), (2, "U-Net")) if v.value & bit]
        raise _lib.FwiError("%s: a bounded wait in the %s kernels gave up (a staging copy did not land); the "
                            "results since the last check are invalid" % (what or "device check", " and ".join(kinds)))


def misfit(data: torch.Tensor, syn: torch.Tensor, adstf: torch.Tensor, nshots: int, nrec: int, nt: int, dt: float,
           stream=None) -> torch.Tensor:
    """Per-shot L2 misfit (FP64) and adjoint source (fwi_misfit)."""
    lib = _lib.load()
    out = torch.zeros(nshots, dtype=torch.float64, device=data.device)
    part = torch.zeros(max(1, nshots * lib.fwi_misfit_partials(nrec, nt)), dtype=torch.float64, device=data.device)
    check(lib.fwi_misfit(ptr(data), ptr(syn), ptr(adstf), ptr(out), ptr(part), nshots, nrec, nt, float(dt),
                         stream_handle(stream)), "fwi_misfit")
    return out


def misfit_tracegrad(data: torch.Tensor, syn: torch.Tensor, grad: torch.Tensor, nshots: int, nrec: int, nt: int,
                     dt: float, stream=None) -> torch.Tensor:
    """Per-shot misfit norm (FP64) and dchi/dsyn in forward time order
    (fwi_misfit_tracegrad)."""
    lib = _lib.load()
    out = torch.zeros(nshots, dtype=torch.float64, device=data.device)
    part = torch.zeros(max(1, nshots * lib.fwi_misfit_partials(nrec, nt)), dtype=torch.float64, device=data.device)
    check(lib.fwi_misfit_tracegrad(ptr(data), ptr(syn), ptr(grad), ptr(out), ptr(part), nshots, nrec, nt, float(dt),
                                   stream_handle(stream)), "fwi_misfit_tracegrad")
    return out


def trace_suffix_sum(g: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Suffix sums along the last (time) axis, FP64-accumulated
    (fwi_trace_suffix_sum): the adjoint displacement at the receivers that
    fwi_run_transposed injects.  out may be g itself."""
    if out is None:
        out = torch.empty_like(g)
    nt = g.shape[-1]
    check(_lib.load().fwi_trace_suffix_sum(ptr(g), ptr(out), g.numel() // max(nt, 1), nt, stream_handle(stream)),
          "fwi_trace_suffix_sum")
    return out


def energy_accumulate(f: torch.Tensor, acc: torch.Tensor, stream=None) -> None:
    """acc += sum over the leading (shot) axis of f^2, FP64 (fwi_energy_accumulate)."""
    field = acc.numel()
    check(_lib.load().fwi_energy_accumulate(ptr(f), f.numel() // max(field, 1), field, ptr(acc), stream_handle(stream)),
          "fwi_energy_accumulate")


def smooth(k: torch.Tensor, grid: Grid, sigma: int, stream=None) -> torch.Tensor:
    """Gaussian smoothing of an FP64 [nx, pitch] kernel into float32 [npt]."""
    out = torch.empty(grid.npt, dtype=torch.float32, device=k.device)
    tmp = torch.empty(grid.npt, dtype=torch.float64, device=k.device)
    check(_lib.load().fwi_smooth(ptr(k), k.shape[-1], ptr(out), grid.nz, ptr(tmp), grid.nx, grid.nz, int(sigma),
                                 stream_handle(stream)), "fwi_smooth")
    return out
