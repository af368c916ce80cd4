"""The ``b200`` solver plugin: a drop-in for seispie's ``fd2d`` solver.

sprun loads a solver as ``getattr(import_module('seispie.solver.' + method),
method)()`` and then sets ``.config`` (a section of strings), ``.path`` (a
dict of absolute paths) and ``.mpi`` before calling ``setup(workflow)``
(scripts/sprun:79-86).  This class keeps that contract and the public method
set and attributes of ``seispie.solver.fd2d.fd2d`` (fd2d.py:110-443):

  setup, import_model, import_sources, import_stations, import_traces,
  run_forward, run_adjoint, run_kernel, compute_misfit, compute_gradient,
  update_model, smooth, export_field, setup_adjoint, clear_kernels,
  clear_wavefields; attributes nx, nz, dx, dz, npt, nt, dt, nsrc, nrec,
  stream (has .synchronize()) and mu (has .copy_to_host(out, stream)).

Differences that a caller can see, all deliberate:
  * All shots of run_kernel are stepped together in one batched launch per
    time step (the reference loops over shots one after another).
  * The P-SV adjoint works (the reference's raises NameError,
    solver.py:324-329) and also yields k_lam and k_rho.
  * Sensitivity kernels accumulate in FP64; the misfit is summed in FP64.
  * Without a GPU the solver refuses to start; there is no CPU path.
"""
from __future__ import annotations

from os import makedirs, path
from time import time

import numpy as np
import torch

from .. import engine
from .._lib import FWI_PSV, FWI_SH, FWI_SPIN
from ..engine import DeviceModel, Grid, ShotBatch


class DeviceArray:
    """A device field with the numba DeviceNDArray method the upper layers
    use: ``copy_to_host(ary, stream)`` (optimize/base.py:59-61)."""

    def __init__(self, tensor: torch.Tensor, nz: int | None = None, stream: torch.cuda.Stream | None = None):
        self.tensor = tensor
        self.nz = nz
        self.stream = stream  # the stream that writes the tensor; reads are ordered after it

    def _flat(self) -> torch.Tensor:
        t = self.tensor
        if t.dim() == 2 and self.nz is not None:
            t = t[:, : self.nz]
        return t.reshape(-1)

    @property
    def size(self) -> int:
        return self._flat().numel()

    def copy_to_host(self, ary: np.ndarray | None = None, stream=None) -> np.ndarray:
        s = stream if isinstance(stream, torch.cuda.Stream) else self.stream
        with torch.cuda.stream(s) if s is not None else _nullctx():
            host = self._flat().to(torch.float32).cpu().numpy()
        if ary is None:
            return host
        ary.reshape(-1)[:] = host
        return ary


def infer_grid(x: np.ndarray, z: np.ndarray, npt):
    """Grid size and spacing from the coordinate arrays of a model file.

    First the reference's formula (fd2d.py:189-196): nx = rint(sqrt(npt*lx/lz)),
    dx = lx/(nx-1) as numpy float32.  It is exact for square grids but not in
    general (1024x512 gives nx = 1025, because lx/lz = (nx-1)/(nz-1), not
    nx/nz); when its nx*nz differs from npt, nz is read from the layout
    instead: the cells k = i*nz + j of row i share one x, so nz is the length
    of the leading run of x == x[0]."""
    lx = x.max() - x.min()
    lz = z.max() - z.min()
    nx = int(np.rint(np.sqrt(npt * lx / lz)))
    nz = int(np.rint(np.sqrt(npt * lz / lx)))
    if nx * nz != npt:
        nz = int(np.argmax(x != x[0])) if np.any(x != x[0]) else int(npt)
        nx = int(npt) // nz
        if nx * nz != npt:
            raise ValueError("model of %d points is not a regular grid" % npt)
    return nx, nz, lx / (nx - 1), lz / (nz - 1)


class _nullctx:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


class b200:
    """B200 FWI solver plugin (drop-in for ``fd2d``)."""

    # ------------------------------------------------------------------ setup
    def setup(self, workflow):
        """fd2d.py:111-120, plus the device and stream of this solver."""
        if not torch.cuda.is_available():
            raise RuntimeError("seispie_b200 needs a CUDA device; there is no CPU path")
        from .. import _lib
        _lib.load()  # fail here, loudly, if the CUDA library is missing
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(self.device)
        self.nt = int(self.config["nt"])
        self.dt = float(self.config["dt"])
        self.sh = 1 if self.config["sh"] == "yes" else 0
        self.psv = 1 if self.config["psv"] == "yes" else 0
        self.spin = 1 if self.config.get("spin", "no") == "yes" else 0
        self.sae = 0
        self.nsa = 0
        self.tile = int(self.config.get("tile", 0))
        self.batch_memory = float(self.config.get("batch_memory_gb", 0)) * 2 ** 30
        self.kernel_rho = self.config.get("kernel_rho", "no") == "yes"
        # model variables of the GPU optimizers: mu alone, as the reference inverts (fd2d.py:442-443),
        # or vp and vs together
        self.invert = self.config.get("invert", "mu")
        if self.invert not in ("mu", "vp_vs"):
            raise ValueError("invert = %r: mu or vp_vs" % self.invert)
        self.model = None

    def _ctx(self):
        return torch.cuda.stream(self.stream)

    @property
    def modes(self):
        """Wave types this configuration runs, in the reference's order."""
        m = []
        if self.sh:
            m.append(FWI_SH)
        if self.psv:
            m.append(FWI_SPIN if self.spin else FWI_PSV)
        return m

    # -------------------------------------------------------------- sources
    def import_sources(self):
        """fd2d.py:122-146: src_id by round-half-even of x/dx and z/dz; the
        Ricker time functions are evaluated on the device (fwi_ricker)."""
        self._drop_graphs()
        src = np.loadtxt(self.path["sources"], ndmin=2)
        self.nsrc = src.shape[0]
        self.src = src
        self.src_id = self._point_ids(src)
        with self._ctx():
            (self.stf_x, self.stf_y, self.stf_z), self._stf_par = engine.ricker_stf(src, self.nt, self.dt,
                                                                                   self.device, self.stream)

    def import_stations(self):
        """fd2d.py:148-165."""
        self._drop_graphs()
        rec = np.loadtxt(self.path["stations"], ndmin=2)
        self.nrec = rec.shape[0]
        self.rec = rec
        self.rec_id = self._point_ids(rec)

    def _point_ids(self, pts: np.ndarray) -> np.ndarray:
        ids = engine.point_ids(pts, self.dx, self.dz, self.nz)
        if len(ids) and (ids.min() < 0 or ids.max() >= self.nx * self.nz):
            raise ValueError("a source or station lies outside the %dx%d grid" % (self.nx, self.nz))
        return ids

    # ---------------------------------------------------------------- model
    def import_model(self, model_true):
        """fd2d.py:167-252: read proc000000_<name>.bin, infer the grid, set
        lambda/mu (vps2lm) and the sponge (set_bound) on the device."""
        self._drop_graphs()
        model = dict()
        model_dir = self.path["model_true"] if model_true else self.path["model_init"]
        names = (["x", "z", "lambda", "mu", "nu", "j", "lambda_c", "mu_c", "nu_c", "rho"] if self.spin
                 else ["x", "z", "vp", "vs", "rho"])
        for name in names:
            filename = path.join(model_dir, "proc000000_" + name + ".bin")
            with open(filename, "rb") as f:
                if not hasattr(self, "npt"):
                    f.seek(0)
                    self.npt = np.fromfile(f, dtype="int32", count=1)
                f.seek(4)
                model[name] = np.fromfile(f, dtype="float32")
        x, z = model["x"], model["z"]
        nx, nz, self.dx, self.dz = infer_grid(x, z, self.npt[0])
        self.nx, self.nz = nx, nz
        self.grid = Grid(nx, nz, float(self.dx), float(self.dz))
        mode = FWI_SPIN if self.spin else (FWI_PSV if self.psv else FWI_SH)
        with self._ctx():
            m = DeviceModel(self.grid, mode, self.dt, self.device, self.stream)
            m.set("rho", model["rho"])
            lib = engine._lib.load()
            if self.spin:
                for dst, src in (("lam", "lambda"), ("mu", "mu"), ("nu", "nu"), ("j", "j"), ("mu_c", "mu_c"),
                                 ("nu_c", "nu_c")):
                    m.set(dst, model[src])
            else:
                m.set("lam", model["vp"])
                m.set("mu", model["vs"])
                engine.check(lib.fwi_vps2lm(engine.ptr(m.lam), engine.ptr(m.mu), engine.ptr(m.rho),
                                            m.lam.numel(), engine.stream_handle(self.stream)), "fwi_vps2lm")
            c = self.config
            engine.check(lib.fwi_set_bound(engine.ptr(m.bound), nx, nz, self.grid.pitch, int(c["abs_width"]),
                                           float(c["abs_alpha"]), c["abs_left"] == "yes", c["abs_right"] == "yes",
                                           c["abs_bottom"] == "yes", c["abs_top"] == "yes",
                                           engine.stream_handle(self.stream)), "fwi_set_bound")
            m.prepare()
        self.model = m
        self.rho = DeviceArray(m.rho, nz, self.stream)
        self.lam = DeviceArray(m.lam, nz, self.stream)
        self.mu = DeviceArray(m.mu, nz, self.stream)
        self.bound = DeviceArray(m.bound, nz, self.stream)
        # fd2d.py:250 tests the raw string, so any non-empty value exports
        if self.config["save_coordinates"]:
            self.export_field(x, "x")
            self.export_field(z, "z")

    def export_field(self, field, name, it=0):
        """fd2d.py:254-261: [int32 npt][float32 field] to output/procIT_name.bin."""
        if isinstance(field, DeviceArray):
            field = field.copy_to_host()
        elif isinstance(field, torch.Tensor):
            field = field.detach().float().cpu().numpy()
        name = "proc%06d_%s" % (it, name)
        with open(self.path["output"] + "/" + name + ".bin", "wb") as f:
            self.npt.tofile(f)
            np.asarray(field, dtype="float32").tofile(f)

    def update_model(self, mu):
        """fd2d.py:442-443: replace mu (only mu) with a fresh upload."""
        with self._ctx():
            self.model.mu.copy_(self.model.pad(np.asarray(mu, dtype="float32")))

    # ------------------------------------------------------------- batching
    def _isrc(self):
        if self.config["combine_sources"] == "yes":
            return -1
        if not hasattr(self, "taskid"):
            raise AttributeError("combine_sources = no needs a task id (set taskid or use run_kernel)")
        return self.taskid

    def _shot_bytes(self, mode, snapshots):
        g = self.grid
        field = g.nx * g.pitch * 4
        ns, nv = engine.NS[mode], engine.NV[mode]
        if snapshots and self._exact(mode):
            from ..adjoint import fixed_bytes
            # checkpoints, segment stores, both batches' wavefields, traces, data and trace gradients
            return fixed_bytes(self.nt, mode, 1, g, self.nrec, overlap=True, density=self._density(mode))
        b = (2 * ns + 3 * nv) * field + 4 * self.nrec * self.nt * nv * 3
        if snapshots:
            b += self.nsa * min(nv, 2) * field * (2 if (mode != FWI_SH and self.kernel_rho) else 1)
        return b

    def _density(self, mode) -> bool:
        """Exact gradient with the density kernel?  Spin always (its dt/j
        kernel shares the stores); SH and P-SV with kernel_rho = yes: without
        it the forward stores no divergence per step (3 instead of 5 fields
        for P-SV), which lengthens the stored tail."""
        return mode == FWI_SPIN or self.kernel_rho

    def _exact(self, mode) -> bool:
        """Gradient by the exact discrete adjoint?  Default: yes for P-SV and
        spin (the reference's adjoint cannot run for them, solver.py:324-329),
        no for SH (its continuous-adjoint kernel equals dt times the exact
        gradient).  Spin has no continuous-adjoint kernel here."""
        g = self.config.get("gradient", "")
        if mode == FWI_SPIN:
            return True
        if g in ("exact", "reference"):
            return g == "exact"
        return mode == FWI_PSV

    def _graph_key(self, mode, shots):
        """What a captured gradient depends on besides the values of the
        model, the observed traces and the time functions: the batch, the
        device buffers the graph reads and the settings of the step loops.
        None when no graph is kept (cuda_graph = no, or batch_memory_gb caps
        the memory of a batch)."""
        if self.config.get("cuda_graph", "yes") != "yes" or self.batch_memory > 0:
            return None
        m = self.model
        names = ("rho", "lam", "mu", "bound", "buo", "nu", "j", "mu_c", "nu_c", "buo_j", "mnc")
        bufs = tuple(getattr(m, n).data_ptr() for n in names if getattr(m, n, None) is not None) + \
            tuple(t.data_ptr() for t in (self.stf_x, self.stf_y, self.stf_z))
        return (mode, tuple(shots), self.config["combine_sources"], self.nt, self.dt, self.tile,
                self._density(mode), tuple(np.asarray(self.src_id).tolist()),
                tuple(np.asarray(self.rec_id).tolist()), bufs)

    def _drop_graphs(self):
        """Release a kept gradient graph and the batch it holds (a new
        model, sources or stations make it stale)."""
        if getattr(self, "_graphs", None):
            self._graphs.clear()
            torch.cuda.empty_cache()

    def _exact_gradient(self, mode, shots, data_of) -> float:
        """Misfit and exact gradient of this process's shots, accumulated in
        the reference's units (dt * dchi/dparam) into k_lam_f64 / k_mu_f64 /
        k_rho_f64; returns the misfit (sum of per-shot, per-component norms).

        With all shots in one batch (the default when they fit), the first
        call computes the gradient step by step and then captures it in CUDA
        graphs (seispie_b200.adjoint.GradientGraph: the forward sweep; the
        misfit step and the backward) that it keeps with the batch's
        buffers; later calls with the same shots, model buffers and settings
        replay them, uploading the observed traces into the graphs' input
        buffers while the forward sweep runs: two launches per gradient, the
        same values bit for bit.  Any other call drops the kept graphs
        first."""
        from ..adjoint import ExactAdjoint, GradientGraph, max_tail_bytes
        key = self._graph_key(mode, shots)
        kept = self.__dict__.setdefault("_graphs", {})
        if key is not None and key in kept:
            return self._replay_gradient(mode, shots, data_of, kept[key])
        self._drop_graphs()  # release a kept batch before this one is sized
        combine = self.config["combine_sources"] == "yes"
        misfit = 0.0
        nrec, nt = self.nrec, self.nt
        for chunk in self._chunks(shots, mode, True):
            n = len(chunk)
            with self._ctx():
                # the last steps keep their per-step stores from the forward sweep (those steps are not
                # recomputed; the gradient is the same): the longest tail that fits 85 % of the free HBM
                # with everything else the gradient holds; not when the configuration caps the memory
                # of a batch
                tail = 0.0
                if self.batch_memory <= 0:
                    tail = max_tail_bytes(nt, mode, n, self.model.grid, 0.85 * self._free_bytes(), nrec,
                                          overlap=True, density=self._density(mode))
                # two segments of per-step stores: the next segment is recomputed on a second stream
                # while this one is transposed
                ea = ExactAdjoint(self.model, nt, self.src_id, lambda s: -1 if combine else chunk[s], n,
                                  self._stf(mode), self.rec_id, tile=self.tile, tail_memory=tail, overlap=True,
                                  density=self._density(mode))
                # the observed traces are stacked into pinned host memory on worker threads while
                # this thread enqueues the forward sweep, then uploaded on a copy stream that the
                # misfit waits for
                staged = self._stage(data_of, chunk, shots)
                tr = ea.forward()
                self.illum_f64 += ea.illum
                grads = [None, None, None]
                uploads = self._upload(staged)
                for slot, (c, lst) in enumerate(data_of):
                    data = uploads[slot]
                    grads[c] = torch.empty(n * nrec * nt, dtype=torch.float32, device=self.device)
                    syn = tr[c].reshape(-1).contiguous()
                    misfit += float(engine.misfit_tracegrad(data, syn, grads[c], n, nrec, nt, self.dt).sum().item())
                    grads[c] = grads[c].view(n, nrec, nt)
                self._accumulate_exact(mode, ea.backward(grads))
                if key is not None and list(chunk) == list(shots):
                    # keep the batch and capture its gradient for the next calls; the uploaded
                    # traces become the graph's input buffers
                    kept[key] = (GradientGraph(ea, self._misfit_step(data_of, uploads, n), warm_up=False), uploads)
                del ea
        return misfit

    def _misfit_step(self, data_of, inputs, n):
        """The misfit step of a captured gradient: trace gradients and
        per-shot misfits of every component slot against the observed
        traces in the device buffers `inputs`."""
        nrec, nt = self.nrec, self.nt

        def between(tr):
            grads, mis = [None, None, None], []
            for slot, (c, lst) in enumerate(data_of):
                g = torch.empty(n * nrec * nt, dtype=torch.float32, device=self.device)
                mis.append(engine.misfit_tracegrad(inputs[slot], tr[c].reshape(-1).contiguous(), g, n, nrec, nt,
                                                   self.dt))
                grads[c] = g.view(n, nrec, nt)
            return grads, mis
        return between

    def _replay_gradient(self, mode, shots, data_of, entry) -> float:
        """A kept gradient graph: the forward sweep replays while the
        observed traces of this call are stacked into pinned memory (worker
        threads) and uploaded into the graph's input buffers (copy stream);
        then the misfit and backward replay and the kernels accumulate as on
        the eager path."""
        gg, inputs = entry
        staged = self._stage(data_of, shots, shots)
        with self._ctx():
            gg.replay_forward()
        copy = self._copy_stream()
        # the previous call's misfit step has read the inputs: that call ended with a host read
        # of its misfit, which followed it on the device
        with torch.cuda.stream(copy):
            for buf, f in zip(inputs, staged):
                buf.copy_(f.result().reshape(buf.shape), non_blocking=True)
        self.stream.wait_stream(copy)
        with self._ctx():
            mis, ks = gg.replay_backward()
            self.illum_f64 += gg.illum
            misfit = 0.0
            for m in mis:
                misfit += float(m.sum().item())
            self._accumulate_exact(mode, ks)
        return misfit

    def _accumulate_exact(self, mode, ks):
        """Add exact-adjoint gradients (ExactAdjoint.backward) to the FP64
        kernels in the reference's units (dt * dchi/dparam)."""
        k_lam, k_mu, k_buo = ks[:3]
        self.k_lam_f64 += self.dt * k_lam
        self.k_mu_f64 += self.dt * k_mu
        if k_buo is not None:
            # buo = dt/rho: dchi/drho = -dchi/dbuo * dt / rho^2
            rho = self.model.rho.double()
            self.k_rho_f64 -= self.dt * k_buo * self.dt / torch.where(rho > 0, rho * rho, torch.ones_like(rho))
        if mode == FWI_SPIN:
            # spin: nu, mu_c and nu_c (both through mnc = mu_c + nu_c), j through dt/j
            k_nu, k_mnc, k_buoj = ks[3:]
            jj = self.model.j.double()
            self.k_nu_f64 += self.dt * k_nu
            self.k_mnc_f64 += self.dt * k_mnc
            self.k_j_f64 -= self.dt * k_buoj * self.dt / torch.where(jj > 0, jj * jj, torch.ones_like(jj))

    def _free_bytes(self) -> int:
        """Free device memory including the blocks torch's caching allocator
        holds unused (those of the previous gradient's buffers), so that
        every call sizes its buffers alike and reuses the cached blocks."""
        free, _ = torch.cuda.mem_get_info(self.device)
        return free + torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)

    def _stage(self, data_of, chunk, shots):
        """Start stacking the observed traces of `chunk` into the pinned
        buffers (one per component slot) on worker threads."""
        return [self._stage_pool().submit(self._stack_pinned, slot, [lst[shots.index(i)] for i in chunk])
                for slot, (c, lst) in enumerate(data_of)]

    def _upload(self, staged):
        """Upload the staged traces on the copy stream; self.stream waits for
        them.  Returns the device tensors, one per component slot."""
        out = []
        for f in staged:
            host = f.result()
            # allocated from the copy stream's pool, so no block that queued forward work still
            # uses can be handed out; recorded on self.stream, which reads it next
            with torch.cuda.stream(self._copy_stream()):
                data = torch.empty(host.shape, dtype=torch.float32, device=self.device)
                data.copy_(host, non_blocking=True)
            data.record_stream(self.stream)
            out.append(data)
        self.stream.wait_stream(self._copy_stream())
        return out

    def _stage_pool(self):
        if getattr(self, "_pool", None) is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=3, thread_name_prefix="seispie_b200_stage")
        return self._pool

    def _copy_stream(self):
        if getattr(self, "_h2d", None) is None:
            self._h2d = torch.cuda.Stream(self.device)
        return self._h2d

    def _stack_pinned(self, slot, arrays):
        """Stack per-shot trace arrays into pinned host buffer `slot` (kept
        and grown across calls).  A buffer is rewritten only after the
        previous call's upload from it has completed: every chunk ends with a
        host read of its misfit, which follows the upload on the device."""
        bufs = self.__dict__.setdefault("_pinned", {})
        n, m = len(arrays), int(np.asarray(arrays[0]).size)
        buf = bufs.get(slot)
        if buf is None or buf.numel() < n * m:
            buf = bufs[slot] = torch.empty(n * m, dtype=torch.float32, pin_memory=True)
        view = buf[:n * m].view(n, m)
        np.stack([np.asarray(a).reshape(-1) for a in arrays], out=view.numpy())
        return view

    def _max_batch(self, mode, snapshots):
        budget = self.batch_memory
        if budget <= 0:
            budget = 0.8 * self._free_bytes()
        return max(1, int(budget // self._shot_bytes(mode, snapshots)))

    def _shots(self):
        """Shots of this process: contiguous shards of range(nsrc) across the
        ranks of self.mpi (the reference gives rank r shot r)."""
        if not self.mpi:
            return list(range(self.nsrc))
        r, n = self.mpi.rank(), self.mpi.size()
        lo, hi = self.nsrc * r // n, self.nsrc * (r + 1) // n
        return list(range(lo, hi))

    def _stf(self, mode):
        return (self.stf_x, self.stf_y, self.stf_z)

    # -------------------------------------------------------------- forward
    def clear_wavefields(self):
        for b in getattr(self, "_fwd_batches", {}).values():
            b.clear()

    def run_forward(self):
        """solver.py:166-287 for one shot set (all sources when
        combine_sources = yes, else source taskid): traces in obs_x/y/z,
        snapshots every save_snapshot steps and output_traces files.

        After setup_adjoint (adjoint_interval set) the forward also keeps
        what run_adjoint needs for this shot, as the reference keeps
        uy_fwd / ux_fwd / uz_fwd: the displacement snapshots of the
        continuous adjoint (SH by default), or the checkpoints of the exact
        adjoint (P-SV and spin by default; no save_snapshot exports then)."""
        isrc = self._isrc()
        sfe = int(self.config["save_snapshot"])
        self._fwd_batches = {}
        self._adjoint_state, self._adj_src = {}, {}
        with self._ctx():
            for mode in self.modes:
                if self.sae and self._exact(mode):
                    self._forward_exact_shot(mode, isrc)
                    continue
                snap = bool(self.sae)
                snapv = snap and mode != FWI_SH and self.kernel_rho
                b = ShotBatch(self.model, 1, self.nt, self.rec_id, sae=self.sae, nsa=self.nsa, snapshots=snap,
                              snap_velocity=snapv, tile=self.tile)
                if snap:
                    self._adjoint_state[mode] = ("snapshots", b)
                inj = engine.injection_lists(1, self.src_id, lambda s: isrc)
                d = b.desc(inj=inj, stf=self._stf(mode))
                b.clear()
                it = 0
                while it < self.nt:
                    n = self.nt - it
                    if sfe:
                        nxt = (it // sfe + 1) * sfe if it > 0 else sfe  # next export step
                        n = min(n, nxt - it + 1)
                    b.run(d, False, it, n)
                    it += n
                    last = it - 1
                    if sfe and last > 0 and last % sfe == 0:
                        names = {FWI_SH: [("vy", "vy")], FWI_PSV: [("vx", "vx"), ("vz", "vz")],
                                 FWI_SPIN: [("vx", "vx"), ("vz", "vz"), ("vy_c", "ry")]}[mode]
                        for f, out in names:
                            self.export_field(b.field(f)[0].reshape(-1), out, last)
                self._fwd_batches[mode] = b
                if mode == FWI_SH:
                    self.obs_y = DeviceArray(b.obs[1], None, self.stream)
                else:
                    self.obs_x = DeviceArray(b.obs[0], None, self.stream)
                    self.obs_z = DeviceArray(b.obs[2], None, self.stream)
                    if mode == FWI_SPIN:
                        self.obs_y = DeviceArray(b.obs[1], None, self.stream)
        self._write_output_traces(isrc)
        engine.check_device(self.stream, "run_forward")

    def _forward_exact_shot(self, mode, isrc):
        """Forward of one shot set with the exact adjoint's checkpoints kept."""
        from ..adjoint import ExactAdjoint
        ea = ExactAdjoint(self.model, self.nt, self.src_id, lambda s: isrc, 1, self._stf(mode), self.rec_id,
                          tile=self.tile, density=self._density(mode))
        tr = ea.forward()
        self.illum_f64 += ea.illum
        self._adjoint_state[mode] = ("exact", ea)
        if mode == FWI_SH:
            self.obs_y = DeviceArray(tr[1].reshape(-1), None, self.stream)
        else:
            self.obs_x = DeviceArray(tr[0].reshape(-1), None, self.stream)
            self.obs_z = DeviceArray(tr[2].reshape(-1), None, self.stream)
            if mode == FWI_SPIN:
                self.obs_y = DeviceArray(tr[1].reshape(-1), None, self.stream)

    def _write_output_traces(self, isrc):
        if "output_traces" in self.path:
            tracedir = self.path["output_traces"]
            i = isrc if isrc >= 0 else 0
            comps = []
            if self.sh:
                comps.append(("uy", self.obs_y))
            if self.psv:
                comps += [("ux", self.obs_x), ("uz", self.obs_z)]
                if self.spin:
                    comps.append(("ry", self.obs_y))
            for name, arr in comps:
                np.save("%s/%s_%06d.npy" % (tracedir, name, i), arr.copy_to_host().reshape([self.nrec, self.nt]))

    # ---------------------------------------------------------------- traces
    def import_traces(self):
        """fd2d.py:354-423: observed traces from raw float32 files
        (vy/vx/vz_%06d.npy), or generated with the current (true) model for
        every shot -- here all shots in one batched forward."""
        shots = self._shots()
        self.syn_x, self.syn_y, self.syn_z = [], [], []
        if "traces" in self.path:
            tracedir = self.path["traces"]
            for i in shots:
                if self.sh:
                    self.syn_y.append(np.fromfile("%s/vy_%06d.npy" % (tracedir, i), dtype="float32"))
                if self.psv:
                    self.syn_x.append(np.fromfile("%s/vx_%06d.npy" % (tracedir, i), dtype="float32"))
                    self.syn_z.append(np.fromfile("%s/vz_%06d.npy" % (tracedir, i), dtype="float32"))
            return
        tracedir = self.path["output"] + "/traces"
        if not self.mpi or self.mpi.rank() == 0:
            print("Generating traces")
            if not path.exists(tracedir):
                makedirs(tracedir)
        if self.mpi:
            self.mpi.sync()
        start = time()
        for mode in self.modes:
            for chunk in self._chunks(shots, mode, False):
                b = self._forward_batch(mode, chunk, snapshots=False)
                for c, lst, nm in ((1, self.syn_y, "vy"), (0, self.syn_x, "vx"), (2, self.syn_z, "vz")):
                    if b.obs[c] is None or (c == 1 and mode == FWI_SPIN):
                        continue
                    with self._ctx():
                        tr = b.traces(c).cpu().numpy()
                    for q, i in enumerate(chunk):
                        out = np.ascontiguousarray(tr[q]).reshape(-1)
                        lst.append(out)
                        out.tofile("%s/%s_%06d.npy" % (tracedir, nm, i))
        if not self.mpi:
            print("Elapsed time: %.2fs" % (time() - start))
            print("")

    def _chunks(self, shots, mode, snapshots):
        m = self._max_batch(mode, snapshots)
        return [shots[q:q + m] for q in range(0, len(shots), m)]

    def _forward_batch(self, mode, chunk, snapshots, snap_velocity=False):
        combine = self.config["combine_sources"] == "yes"
        with self._ctx():
            b = ShotBatch(self.model, len(chunk), self.nt, self.rec_id, sae=self.sae, nsa=self.nsa,
                          snapshots=snapshots, snap_velocity=snap_velocity, tile=self.tile)
            inj = engine.injection_lists(len(chunk), self.src_id, lambda s: -1 if combine else chunk[s])
            d = b.desc(inj=inj, stf=self._stf(mode))
            b.clear()
            b.run(d, False, 0, self.nt)
        return b

    # --------------------------------------------------------------- adjoint
    def setup_adjoint(self):
        """fd2d.py:263-301: adjoint interval, snapshot count, kernels and the
        smoothing width.  Snapshots live in HBM (allocated per batch)."""
        self.sae = int(self.config["adjoint_interval"])
        self.nsa = int(self.nt / self.sae)
        self.sigma = int(self.config["smooth"])
        g = self.grid
        with self._ctx():
            self.k_lam_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            self.k_mu_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            self.k_rho_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            self.illum_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            # spin gradients (dt * dchi/dnu, dt * dchi/d(mu_c) = dt * dchi/d(nu_c), dt * dchi/dj)
            self.k_nu_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            self.k_mnc_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
            self.k_j_f64 = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)

    def clear_kernels(self):
        with self._ctx():
            for k in (self.k_lam_f64, self.k_mu_f64, self.k_rho_f64, self.illum_f64, self.k_nu_f64, self.k_mnc_f64,
                      self.k_j_f64):
                k.zero_()

    def illumination_device(self):
        """Source illumination of the last exact-adjoint gradient (squared
        particle velocity summed over checkpoints and shots), float32 CUDA
        vector of npt, or None when the gradient did not come from the exact
        adjoint.  No counterpart in the reference; read by the learned
        preconditioner."""
        if not getattr(self, "_illum_valid", False):
            return None
        with self._ctx():
            out = self.illum_f64[:, : self.nz].float().reshape(-1).clone()
        self.stream.synchronize()
        return out

    def _compute_misfit(self, comp, h_syn):
        """fd2d.py:303-309: the L2 misfit norm of component comp ('x', 'y' or
        'z') of the last run_forward against the observed traces h_syn, and
        that component's adjoint source for run_adjoint -- time-reversed
        2 taper^2 (d - s) for the continuous adjoint (waveform.py:24-34), the
        trace gradient in forward time for the exact adjoint."""
        c = "xyz".index(comp)
        nrec, nt = self.nrec, self.nt
        obs = getattr(self, "obs_" + comp).tensor.reshape(-1)
        exact = any(k == "exact" and c in self._comps(mode) for mode, (k, _) in self._adjoint_state.items())
        with self._ctx():
            data = torch.as_tensor(np.ascontiguousarray(h_syn, dtype=np.float32).reshape(-1)).to(self.device)
            src = torch.empty(nrec * nt, dtype=torch.float32, device=self.device)
            if exact:
                m = engine.misfit_tracegrad(data, obs, src, 1, nrec, nt, self.dt, self.stream)
            else:
                m = engine.misfit(data, obs, src, 1, nrec, nt, self.dt, self.stream)
            self._adj_src[c] = src
            misfit = float(m.sum().item())
        return misfit

    @staticmethod
    def _comps(mode):
        """Component slots whose traces enter the misfit of a wave type."""
        return (1,) if mode == FWI_SH else (0, 2)

    def run_adjoint(self):
        """solver.py:290-321 for the shot of the last run_forward, after
        _compute_misfit of its components: the adjoint run whose kernels are
        added to k_mu (and k_lam, k_rho) -- the snapshot-correlation adjoint
        of the reference for SH, the exact transposed step for P-SV and spin
        (the reference's P-SV branch cannot run, solver.py:324-329)."""
        state = getattr(self, "_adjoint_state", None)
        if not state:
            raise RuntimeError("run_adjoint needs setup_adjoint, then run_forward")
        nrec, nt = self.nrec, self.nt
        with self._ctx():
            for mode, (kind, obj) in state.items():
                comps = self._comps(mode)
                missing = [c for c in comps if c not in self._adj_src]
                if missing:
                    raise RuntimeError("run_adjoint: _compute_misfit('%s') first" % "xyz"[missing[0]])
                if kind == "exact":
                    grads = [self._adj_src[c].view(1, nrec, nt) if c in comps else None for c in range(3)]
                    self._accumulate_exact(mode, obj.backward(grads))
                else:
                    b = obj
                    adstf = [self._adj_src.get(c) if c in comps else None for c in range(3)]
                    snapv = mode != FWI_SH and self.kernel_rho
                    kern = (None, self.k_mu_f64, None) if mode == FWI_SH else \
                        (self.k_lam_f64, self.k_mu_f64, self.k_rho_f64 if snapv else None)
                    d = b.desc(inj=engine.adjoint_injection_lists(1, self.rec_id), stf=adstf, record=False,
                               kernels=kern)
                    b.clear()
                    b.run(d, True, 0, nt)
        self._adjoint_state, self._adj_src = {}, {}
        self._illum_valid = all(self._exact(m) for m in self.modes)
        engine.check_device(self.stream, "run_adjoint")

    def run_kernel(self, adj):
        """solver.py:332-404, all shots of this process batched: forward with
        snapshots, misfit and adjoint source, adjoint with interaction, then
        the cross-rank sum and the Gaussian smoothing of k_mu."""
        if not self.mpi:
            print("Computing kernels" if adj else "Computing misfit")
        self.setup_adjoint()
        self.clear_kernels()
        self._illum_valid = bool(adj) and all(self._exact(m) for m in self.modes)
        shots = self._shots()
        misfit = 0.0
        data_of = {FWI_SH: [(1, self.syn_y)], FWI_PSV: [(0, self.syn_x), (2, self.syn_z)],
                   FWI_SPIN: [(0, self.syn_x), (2, self.syn_z)]}
        for mode in self.modes:
            snapv = adj and mode != FWI_SH and self.kernel_rho
            if adj and self._exact(mode):
                misfit += self._exact_gradient(mode, shots, data_of[mode])
                continue
            for chunk in self._chunks(shots, mode, adj):
                staged = self._stage(data_of[mode], chunk, shots)  # on worker threads during the forward
                b = self._forward_batch(mode, chunk, snapshots=bool(adj), snap_velocity=snapv)
                n, nrec, nt = len(chunk), self.nrec, self.nt
                with self._ctx():
                    adstf = [None, None, None]
                    uploads = self._upload(staged)
                    for slot, (c, lst) in enumerate(data_of[mode]):
                        data = uploads[slot]
                        adstf[c] = torch.empty(n * nrec * nt, dtype=torch.float32, device=self.device)
                        m = engine.misfit(data, b.obs[c], adstf[c], n, nrec, nt, self.dt)
                        misfit += float(m.sum().item())
                    if adj:
                        kern = (None, self.k_mu_f64, None) if mode == FWI_SH else \
                               (self.k_lam_f64, self.k_mu_f64, self.k_rho_f64 if snapv else None)
                        d = b.desc(inj=engine.adjoint_injection_lists(n, self.rec_id), stf=adstf, record=False,
                                   kernels=kern)
                        b.clear()
                        b.run(d, True, 0, nt)
                del b
        # every kernel of this gradient has run its bounded waits to the end, or the call fails here
        engine.check_device(self.stream, "run_kernel")
        if self.mpi:
            misfit = self._mpi_sum_misfit(misfit)
            self._mpi_sum_kernels()
        if adj:
            with self._ctx():
                self.k_mu = DeviceArray(engine.smooth(self.k_mu_f64, self.grid, self.sigma), None, self.stream)
                self.k_lam = DeviceArray(self.k_lam_f64, self.nz, self.stream)
                self.k_rho = DeviceArray(self.k_rho_f64, self.nz, self.stream)
        if not self.mpi:
            print("  misfit = %.2f" % misfit)
        if adj:
            return misfit, self.k_mu, self.mu
        return misfit

    def _mpi_sum_misfit(self, misfit):
        out = np.zeros(1, dtype="float64")
        self.mpi.sum(np.array([misfit], dtype="float64"), out)
        return float(out[0])

    def _mpi_sum_kernels(self):
        """Cross-rank sum of the FP64 kernels (replaces the file exchange of
        solver.py:380-393, which also counted the local kernel twice)."""
        if hasattr(self.mpi, "allreduce_tensor"):
            self.stream.synchronize()
            for k in self._summed_fields():
                self.mpi.allreduce_tensor(k)
        else:
            for k in self._summed_fields():
                host = k.cpu().numpy()
                out = np.zeros_like(host)
                self.mpi.sum(host, out)
                k.copy_(torch.from_numpy(out))

    def _summed_fields(self):
        return (self.k_lam_f64, self.k_mu_f64, self.k_rho_f64, self.illum_f64, self.k_nu_f64, self.k_mnc_f64,
                self.k_j_f64)

    def compute_misfit(self):
        return self.run_kernel(0)

    def compute_gradient(self):
        """fd2d.py:428-437: (smoothed k_mu, misfit, mu) as host float32."""
        misfit, kernel, model = self.run_kernel(1)
        out_k = kernel.copy_to_host(stream=self.stream)
        out_m = model.copy_to_host(stream=self.stream)
        self.stream.synchronize()
        return out_k, misfit, out_m

    def compute_gradient_device(self):
        """compute_gradient without leaving the device: (smoothed gradient,
        misfit, model) as float32 CUDA vectors (the GPU optimizers' entry).
        invert = mu: k_mu and mu, npt each.  invert = vp_vs: [vp; vs] (2 npt)
        and its gradient from the exact kernels by the chain rule,
        dchi/dvp = 2 rho vp k_lam and dchi/dvs = 2 rho vs (k_mu - 2 k_lam),
        each smoothed like k_mu."""
        misfit, kernel, model = self.run_kernel(1)
        with self._ctx():
            if self.invert == "mu":
                g = kernel.tensor.reshape(-1).clone()
                m = model._flat().clone()
            else:
                nz = self.nz
                rho = self.model.rho.double()
                vp, vs = self._velocities()
                g_vp = 2.0 * rho * vp.double() * self.k_lam_f64
                g_vs = 2.0 * rho * vs.double() * (self.k_mu_f64 - 2.0 * self.k_lam_f64)
                g = torch.cat([engine.smooth(g_vp, self.grid, self.sigma, self.stream),
                               engine.smooth(g_vs, self.grid, self.sigma, self.stream)])
                m = torch.cat([vp[:, :nz].reshape(-1), vs[:, :nz].reshape(-1)]).clone()
        self.stream.synchronize()
        return g, misfit, m

    def _velocities(self):
        """vp, vs ([nx, pitch] float32) of the current lam, mu, rho
        (lm2vps, fd2d.py:36-44)."""
        vp, vs = self.model.lam.clone(), self.model.mu.clone()
        engine.check(engine._lib.load().fwi_lm2vps(engine.ptr(vp), engine.ptr(vs), engine.ptr(self.model.rho),
                                                   vp.numel(), engine.stream_handle(self.stream)), "fwi_lm2vps")
        return vp, vs

    def update_model_device(self, m: torch.Tensor):
        """update_model from a float32 CUDA vector: mu (npt), or [vp; vs]
        (2 npt) converted to lam and mu on the device (vps2lm,
        fd2d.py:21-33)."""
        torch.cuda.current_stream().synchronize()
        nx, nz, npt = self.nx, self.nz, self.nx * self.nz
        with self._ctx():
            if self.invert == "mu":
                self.model.mu[:, :nz].copy_(m.reshape(nx, nz))
            else:
                self.model.lam[:, :nz].copy_(m[:npt].reshape(nx, nz))
                self.model.mu[:, :nz].copy_(m[npt:].reshape(nx, nz))
                engine.check(engine._lib.load().fwi_vps2lm(engine.ptr(self.model.lam), engine.ptr(self.model.mu),
                                                           engine.ptr(self.model.rho), self.model.lam.numel(),
                                                           engine.stream_handle(self.stream)), "fwi_vps2lm")

    def export_model(self, m, it):
        """Write an optimizer model vector as the reference's model files:
        mu, or vp and vs (fd2d.py:254-261)."""
        m = m.detach().float().cpu().numpy() if isinstance(m, torch.Tensor) else np.asarray(m, np.float32)
        npt = self.nx * self.nz
        if self.invert == "mu":
            self.export_field(m[:npt], "mu", it)
        else:
            self.export_field(m[:npt], "vp", it)
            self.export_field(m[npt:], "vs", it)

    def model_vector_device(self):
        """The optimizer's model vector of the current model (float32 CUDA)."""
        with self._ctx():
            if self.invert == "mu":
                m = self.model.mu[:, : self.nz].reshape(-1).clone()
            else:
                vp, vs = self._velocities()
                m = torch.cat([vp[:, : self.nz].reshape(-1), vs[:, : self.nz].reshape(-1)])
        self.stream.synchronize()
        return m

    def smooth(self, data):
        """fd2d.py:349-352: Gaussian smoothing of a device field (FP64
        [nx, pitch] tensor, or a DeviceArray); returns a float32 DeviceArray."""
        t = data.tensor if isinstance(data, DeviceArray) else data
        with self._ctx():
            if t.dim() == 1:
                g = self.grid
                pad = torch.zeros((g.nx, g.pitch), dtype=torch.float64, device=self.device)
                pad[:, : g.nz] = t.view(g.nx, g.nz).double()
                t = pad
            return DeviceArray(engine.smooth(t.double(), self.grid, int(self.config["smooth"])), None, self.stream)
