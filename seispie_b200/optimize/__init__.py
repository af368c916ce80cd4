"""GPU optimizers with the step logic of seispie/optimize (base.py, gd.py,
cg.py, lbfgs.py, sgd.py): the model, gradient, directions and L-BFGS pairs
stay on the device as float32 vectors; dot products, max-norms and updates
are FP64 GPU kernels (VecOps); scalar decisions are host code as in the
reference.  The solver must be the b200 plugin (device-side
compute_gradient_device / update_model_device)."""
from __future__ import annotations

from time import time

import numpy as np

from .line_search import backtrack, bracket
from .vec import VecOps


class base:
    """optimize/base.py:4-69."""

    def setup(self, workflow):
        raise NotImplementedError

    def compute_direction(self):
        raise NotImplementedError

    def line_search(self, misfit):
        raise NotImplementedError

    def restart_search(self):
        raise NotImplementedError

    def run(self):
        solver = self.solver
        niter = int(self.config["niter"])
        start = time()
        misfits = []
        head = 0 if (self.mpi and self.mpi.rank()) else 1
        self.history = []
        ref = None
        for i in range(niter):
            if head:
                print("Iteration %d" % (i + 1))
            self.g_new, misfit, self.m_new = solver.compute_gradient_device()
            if head:
                if i > 0:
                    solver.export_model(self.m_new, i - 1)
                else:
                    ref = misfit
                misfits.append(misfit / ref)
            self.history.append(dict(iteration=i, misfit=misfit, t=time() - start))
            self.p_new = self.compute_direction()
            self.m_old, self.p_old, self.g_old = self.m_new, self.p_new, self.g_new
            if self.line_search(misfit) < 0:
                if head:
                    print("Line search failed")
                    break
            if head:
                print("")
        misfit = solver.compute_misfit()
        self.history.append(dict(iteration=niter, misfit=misfit, t=time() - start))
        if head:
            misfits.append(misfit / ref)
            solver.export_model(solver.model_vector_device(), niter)
            print("Misfits:")
            for m in misfits:
                print("  %.4f" % m)
            print("")
            print("Elapsed time: %.2fs" % (time() - start))
        self.misfits = misfits


class cg(base):
    """Polak-Ribiere conjugate gradient (cg.py:5-49)."""

    def setup(self, workflow):
        self.solver = workflow.solver
        self.ops = VecOps(self.solver.device)
        self.bracket = bracket(workflow.solver, self.config, self.ops)
        self.bracket.head = 0 if (self.mpi and self.mpi.rank()) else 1

    def line_search(self, misfit):
        return self.bracket.run(self.m_new, self.g_new, self.p_new, misfit)

    def restart_search(self):
        self.bracket.restart()

    def pollak(self, g_new, g_old):
        d = self.ops.axpby(1.0, g_new, -1.0, g_old)
        return self.ops.dot(g_new, d) / self.ops.dot(g_old, g_old)

    def fletcher(self, g_new, g_old):
        return self.ops.dot(g_new, g_new) / self.ops.dot(g_old, g_old)

    def compute_direction(self):
        if not hasattr(self, "g_old"):
            return self.ops.axpby(-1.0, self.g_new)
        beta = self.pollak(self.g_new, self.g_old)
        p_new = self.ops.axpby(-1.0, self.g_new, beta, self.p_old)
        if self.ops.dot(p_new, self.g_new) > 0:
            print("  restarting CG: not descent")
            self.restart_search()
            return self.ops.axpby(-1.0, self.g_new)
        return p_new


class gd(cg):
    """Steepest descent (gd.py:3-5)."""

    def compute_direction(self):
        return self.ops.axpby(-1.0, self.g_new)


class lbfgs(cg):
    """Two-loop L-BFGS with the backtracking line search (lbfgs.py:5-59)."""

    def setup(self, workflow):
        self.solver = workflow.solver
        self.ops = VecOps(self.solver.device)
        self.bracket = backtrack(workflow.solver, self.config, self.ops)
        self.bracket.head = 0 if (self.mpi and self.mpi.rank()) else 1
        self.lbfgs_s, self.lbfgs_y = [], []
        self.lbfgs_mem = int(self.config["lbfgs_mem"])

    def restart_search(self):
        super().restart_search()
        self.lbfgs_s, self.lbfgs_y = [], []

    def compute_direction(self):
        ops, g_new = self.ops, self.g_new
        if not hasattr(self, "g_old"):
            return ops.axpby(-1.0, g_new)
        self.lbfgs_s.insert(0, ops.axpby(1.0, self.m_new, -1.0, self.m_old))
        self.lbfgs_y.insert(0, ops.axpby(1.0, g_new, -1.0, self.g_old))
        if len(self.lbfgs_s) > self.lbfgs_mem:
            self.lbfgs_s.pop()
            self.lbfgs_y.pop()
        n = len(self.lbfgs_s)
        rh, al = np.zeros(n), np.zeros(n)
        q = g_new.clone()
        for i in range(n):
            rh[i] = 1 / ops.dot(self.lbfgs_y[i], self.lbfgs_s[i])
            al[i] = rh[i] * ops.dot(self.lbfgs_s[i], q)
            ops.axpby(1.0, q, -al[i], self.lbfgs_y[i], out=q)
        ops.axpby(ops.dot(self.lbfgs_y[0], self.lbfgs_s[0]) / ops.dot(self.lbfgs_y[0], self.lbfgs_y[0]), q, out=q)
        for i in range(n - 1, -1, -1):
            be = rh[i] * ops.dot(self.lbfgs_y[i], q)
            ops.axpby(1.0, q, al[i] - be, self.lbfgs_s[i], out=q)
        if self.bracket.angle(g_new, q) >= np.pi / 2:
            print("  restarting LBFGS: not descent")
            self.restart_search()
            return ops.axpby(-1.0, g_new)
        return ops.axpby(-1.0, q)


class sgd(base):
    """sgd.py:5-57 is a verbatim copy of base.run; kept as an alias."""


from .learned import lbfgs_learned  # noqa: E402  (needs lbfgs above)

__all__ = ["base", "cg", "gd", "lbfgs", "lbfgs_learned", "sgd", "bracket", "backtrack", "VecOps"]
