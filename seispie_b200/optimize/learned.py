"""L-BFGS with a learned preconditioner (``[optimize] method = lbfgs_learned``).

The step logic is the reference's L-BFGS (optimize/lbfgs.py:5-59) with its
backtracking line search; on top of it:

* ``unet_weights = <file.npz>``: in the first ``learned_iterations``
  iterations (default: the number stored with the weights, else
  ``lbfgs_mem``: while the L-BFGS memory is still short) the U-Net (seispie_b200.unet) maps (gradient, source illumination,
  model) to an update direction, scaled to the max-norm of the L-BFGS
  direction.  It is used only if it is a descent direction (g.p < 0) and its
  line search succeeds; otherwise the plain L-BFGS direction is searched
  from a clean line-search history.  The L-BFGS memory is built from model
  and gradient differences either way, so the later L-BFGS iterations start
  from the learned steps' curvature pairs.
* ``record_pairs = <file.npz>``: stores, per iteration, the gradient, the
  illumination, the model and the accepted update m_{k+1} - m_k -- the
  training pairs of the preconditioner.

Without either key it is plain L-BFGS.  Needs the b200 solver with the exact
adjoint gradient (the default for P-SV), which provides the illumination.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lbfgs


class lbfgs_learned(lbfgs):
    def setup(self, workflow):
        super().setup(workflow)
        if getattr(self.solver, "invert", "mu") != "mu":
            raise ValueError("the learned preconditioner maps mu gradients: use invert = mu")
        self.pre = None
        path = self.config.get("unet_weights", "") if hasattr(self.config, "get") else ""
        if path:
            from ..learned import Preconditioner
            self.pre = Preconditioner.load(path, self.solver.device)
        self.record = self.config.get("record_pairs", "") if hasattr(self.config, "get") else ""
        self.pairs = []
        self.learned_accepted = 0
        self.learned_rejected = 0
        get = self.config.get if hasattr(self.config, "get") else (lambda k, d=None: d)
        hint = self.pre.learned_iterations if self.pre is not None else None
        self.learned_iterations = int(get("learned_iterations", str(hint or self.lbfgs_mem)))
        self.iteration = 0

    def compute_direction(self):
        p_plain = super().compute_direction()
        self.p_plain, self.used_learned = p_plain, False
        self.illum = self.solver.illumination_device()
        self.iteration += 1
        if self.pre is None or self.illum is None or self.iteration > self.learned_iterations:
            return p_plain
        p = self.pre.direction(self.g_new, self.illum, self.m_new, self.solver.nx, self.solver.nz,
                               self.ops.absmax(p_plain))
        if not self.ops.dot(self.g_new, p) < 0:
            self.learned_rejected += 1
            return p_plain
        self.used_learned = True
        return p

    def line_search(self, misfit):
        if self.used_learned:
            status = self.bracket.run(self.m_new, self.g_new, self.p_new, misfit, allow_restart=False)
            if status >= 0:
                self.learned_accepted += 1
                self._record()
                return status
            self.learned_rejected += 1
            self.bracket.restart()
            self.p_new = self.p_old = self.p_plain
        status = self.bracket.run(self.m_new, self.g_new, self.p_new, misfit)
        if status >= 0:
            self._record()
        return status

    def _record(self):
        if not self.record or self.illum is None:
            return
        torch.cuda.synchronize()
        m_after = self.solver.mu._flat().clone()
        d = self.ops.axpby(1.0, m_after, -1.0, self.m_new)
        self.pairs.append(tuple(t.detach().cpu().numpy().astype(np.float32)
                                for t in (self.g_new, self.illum, self.m_new, d)))

    def run(self):
        super().run()
        if self.record and self.pairs:
            g, i, m, d = (np.stack(x) for x in zip(*self.pairs))
            np.savez(self.record, g=g, illum=i, m=m, d=d, nx=self.solver.nx, nz=self.solver.nz)
