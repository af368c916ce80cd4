"""Line searches with the step logic of seispie/optimize/line_search/*.py
(bracket.py:3-164, backtrack.py:4-27), on device vectors.

The trial-step arithmetic (history, bracketing test, parabolic fit,
backtracking) is scalar and runs on the host exactly as in the reference;
the model updates m + alpha*p, dot products and max-norms run on the GPU in
FP64 (VecOps).  The solver must offer update_model_device(m) and
compute_misfit().
"""
from __future__ import annotations

import numpy as np

from .vec import VecOps


class bracket:
    """Bracketing line search with a parabolic fit (bracket.py)."""

    def __init__(self, solver, config, ops: VecOps):
        self.solver, self.ops = solver, ops
        self.ls_lens, self.ls_vals, self.ls_gtg, self.ls_gtp = [], [], [], []
        self.ls_step = int(config["ls_step"])
        self.ls_step_max = float(config["ls_step_max"])
        self.ls_step_init = float(config["ls_step_init"])
        self.ls_thresh = float(config.get("ls_thresh", 1.2))  # parsed, unused, as bracket.py:15
        self.head = 1

    def restart(self):
        self.ls_lens, self.ls_vals, self.ls_gtg, self.ls_gtp = [], [], [], []

    def angle(self, x, y) -> float:
        """bracket.py:23-30 with FP64 GPU dots."""
        xy, xx, yy = self.ops.dot(x, y), self.ops.dot(x, x), self.ops.dot(y, y)
        ang = xy / (xx * yy) ** 0.5
        if abs(ang) > 1:
            ang /= abs(ang)
        return float(np.arccos(ang))

    def _trial(self, m_new, p_new, alpha):
        self.solver.update_model_device(self.ops.axpby(1.0, m_new, alpha, p_new))

    def run(self, m_new, g_new, p_new, f, allow_restart: bool = True) -> int:
        """bracket.py:32-81.  allow_restart = False returns the failure status
        instead of restarting the search along the same direction (used when
        a caller has another direction to fall back to).  The reference
        restarts by recursing without limit; a restarted search repeats the
        same trial steps, so a second failure is returned instead of
        recursing until the interpreter's stack is exhausted."""
        if self.head:
            print("  step 1")
        ops = self.ops
        norm_m, norm_p = ops.absmax(m_new), ops.absmax(p_new)
        gtg, gtp = ops.dot(g_new, g_new), ops.dot(g_new, p_new)
        step_max = self.ls_step_max * norm_m / norm_p
        step_count = 0
        self.ls_lens.append(0)
        self.ls_vals.append(f)
        self.ls_gtg.append(gtg)
        self.ls_gtp.append(gtp)
        if self.ls_step_init and len(self.ls_lens) <= 1:
            alpha = self.ls_step_init * norm_m / norm_p
        else:
            alpha, status = self.calculate_step(step_count, step_max)
        while True:
            self._trial(m_new, p_new, alpha)
            self.ls_lens.append(alpha)
            self.ls_vals.append(self.solver.compute_misfit())
            step_count += 1
            alpha, status = self.calculate_step(step_count, step_max)
            if self.head:
                print("  step %d" % (step_count + 1))
            if status > 0:
                self._trial(m_new, p_new, alpha)
                return status
            if status < 0:
                self.solver.update_model_device(m_new)
                neg_g = ops.axpby(-1.0, g_new)
                if self.angle(p_new, neg_g) < 1e-3 or not allow_restart:
                    return status
                if self.head:
                    print("  restarting line search")
                self.restart()
                return self.run(m_new, g_new, p_new, f, allow_restart=False)

    def get_history(self, i):
        """bracket.py:83-89."""
        k = len(self.ls_lens)
        x = np.array(self.ls_lens[k - i - 1:k])
        f = np.array(self.ls_vals[k - i - 1:k])
        order = abs(x).argsort()
        return x[order], f[order], sum(np.array(self.ls_lens) == 0) - 1

    def calculate_step(self, step_count, step_max):
        """bracket.py:91-132."""
        x, f, update_count = self.get_history(step_count)
        if step_count == 0:
            if update_count == 0:
                alpha, status = 1 / self.ls_gtg[-1], 0
            else:
                idx = np.argmin(self.ls_vals[:-1])
                alpha, status = self.ls_lens[idx] * self.ls_gtp[-2] / self.ls_gtp[-1], 0
        elif self.check_bracket(x, f):
            if self.good_enough(x, f):
                alpha, status = x[f.argmin()], 1
            else:
                alpha, status = self.polyfit(x, f), 0
        elif step_count <= self.ls_step:
            if all(f <= f[0]):
                alpha, status = 1.618034 * x[step_count], 0
            else:
                slope = self.ls_gtp[-1] / self.ls_gtg[-1]
                alpha, status = self.backtrack(f[0], slope, x[1], f[1], 0.1, 0.5), 0
        else:
            alpha, status = 0, -1
        if alpha > step_max:
            if step_count == 0:
                alpha, status = 0.618034 * step_max, 0
            else:
                alpha, status = step_max, 1
        return alpha, status

    def check_bracket(self, x, f):
        imin, fmin = f.argmin(), f.min()
        return 1 if (fmin < f[0]) and any(f[imin:] > fmin) else 0

    def good_enough(self, x, f):
        if not self.check_bracket(x, f):
            return 0
        x0 = self.polyfit(x, f)
        return 1 if any(np.abs(np.log10(x[1:] / x0)) < np.log10(1.2)) else 0

    def polyfit(self, x, f):
        i = np.argmin(f)
        p = np.polyfit(x[i - 1:i + 2], f[i - 1:i + 2], 2)
        if p[0] > 0:
            return -p[1] / (2 * p[0])
        raise RuntimeError("line search: parabolic fit is not convex (bracket.polyfit)")

    def backtrack(self, f0, g0, x1, f1, b1, b2):
        x2 = -g0 * x1 ** 2 / (2 * (f1 - f0 - g0 * x1))
        if x2 > b2 * x1:
            x2 = b2 * x1
        elif x2 < b1 * x1:
            x2 = b1 * x1
        return x2


class backtrack(bracket):
    """backtrack.py:4-27 (the comparison of step_count with step_max at
    backtrack.py:19 is the reference's and is kept)."""

    def calculate_step(self, step_count, step_max):
        x, f, update_count = self.get_history(step_count)
        if update_count == 0:
            return super().calculate_step(step_count, step_max)
        if step_count == 0:
            return min(1.0, step_max), 0
        if f.min() < f[0]:
            return x[f.argmin()], 1
        if step_count <= step_max:
            slope = self.ls_gtp[-1] / self.ls_gtg[-1]
            return self.backtrack(f[0], slope, x[1], f[1], 0.1, 0.5), 0
        return 0, -1
