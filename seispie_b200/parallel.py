"""The reference's ``mpi`` object (seispie/tools/mpi.py:3-14) over
torch.distributed: one process per GPU, NCCL for device tensors (gloo on
CPU-only hosts).

Shots are the unit of parallelism (solver.py:352-353): each rank runs a
contiguous block of shots and the ranks sum their FP64 sensitivity kernels
and misfits -- one all-reduce per gradient, replacing the reference's
exchange through files (solver.py:380-393).
"""
from __future__ import annotations

import datetime
import os

import numpy as np
import torch
import torch.distributed as dist


class TorchMPI:
    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        if not dist.is_initialized():
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            kw = {}
            if backend == "nccl":
                local = int(os.environ.get("LOCAL_RANK", "0"))
                torch.cuda.set_device(local)
                kw["device_id"] = torch.device("cuda", local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
        self.backend = dist.get_backend()

    def rank(self) -> int:
        return dist.get_rank()

    def size(self) -> int:
        return dist.get_world_size()

    def sync(self) -> None:
        dist.barrier()

    def _device(self):
        return torch.device("cuda", torch.cuda.current_device()) if self.backend == "nccl" else torch.device("cpu")

    def sum(self, data, out) -> None:
        """Allreduce(SUM) of a numpy array into out (mpi.py:13-14), in FP64."""
        t = torch.as_tensor(np.asarray(data, dtype=np.float64)).to(self._device())
        dist.all_reduce(t)
        np.asarray(out).reshape(-1)[:] = t.cpu().numpy().reshape(-1)

    def allreduce_tensor(self, t: torch.Tensor) -> None:
        """In-place sum of a tensor on the backend's device."""
        dist.all_reduce(t)

    def close(self) -> None:
        if dist.is_initialized():
            dist.destroy_process_group()


def shard(n: int, rank: int, size: int) -> range:
    """Contiguous block of range(n) owned by rank."""
    return range(n * rank // size, n * (rank + 1) // size)
