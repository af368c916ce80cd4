"""Model-sized float32 vectors on the device and the FP64 operations the
optimizers need, all through libseispie_b200 (fwi_dot, fwi_absmax,
fwi_axpby).  Scalars come back to the host because the step logic that
consumes them (line search, restarts) is scalar host code, as in the
reference (seispie/optimize/*)."""
from __future__ import annotations

import torch

from .. import _lib
from ..engine import stream_handle


class VecOps:
    def __init__(self, device):
        self.device = device
        n = int(_lib.load().fwi_reduce_partials())
        self._pd = torch.empty(n, dtype=torch.float64, device=device)
        self._pf = torch.empty(n, dtype=torch.float32, device=device)
        self._od = torch.empty(1, dtype=torch.float64, device=device)
        self._of = torch.empty(1, dtype=torch.float32, device=device)

    def dot(self, x: torch.Tensor, y: torch.Tensor) -> float:
        _lib.check(_lib.load().fwi_dot(x.data_ptr(), y.data_ptr(), x.numel(), self._od.data_ptr(),
                                       self._pd.data_ptr(), stream_handle(None)), "fwi_dot")
        return float(self._od.item())

    def absmax(self, x: torch.Tensor) -> float:
        _lib.check(_lib.load().fwi_absmax(x.data_ptr(), x.numel(), self._of.data_ptr(), self._pf.data_ptr(),
                                          stream_handle(None)), "fwi_absmax")
        return float(self._of.item())

    def axpby(self, a: float, x: torch.Tensor, b: float = 0.0, y: torch.Tensor | None = None,
              out: torch.Tensor | None = None) -> torch.Tensor:
        """a*x + b*y (FP64 arithmetic, float32 result); new tensor unless out."""
        o = torch.empty_like(x) if out is None else out
        _lib.check(_lib.load().fwi_axpby(o.data_ptr(), float(a), x.data_ptr(), float(b),
                                         None if y is None else y.data_ptr(), x.numel(), stream_handle(None)),
                   "fwi_axpby")
        return o
