"""seispie's on-disk formats.

* Model / field files ``procIIIIII_<name>.bin``: int32 npt, then npt float32
  in the reference's cell order k = i*nz + j (fd2d.py:174-182, 254-261).
* Observed traces ``{vx,vy,vz}_IIIIII.npy``: raw float32 (no .npy header),
  receiver-major [nrec*nt] (fd2d.py:372-376, 406-417).
* Output traces ``{ux,uy,uz,ry}_IIIIII.npy``: real .npy of shape [nrec, nt]
  (solver.py:263-287).
"""
from __future__ import annotations

import os

import numpy as np


def write_field(path: str, field: np.ndarray, npt: int | None = None) -> None:
    """[int32 npt][float32 field] (export_field, fd2d.py:254-261)."""
    f32 = np.asarray(field, dtype="float32").ravel()
    with open(path, "wb") as f:
        np.array([f32.size if npt is None else npt], dtype="int32").tofile(f)
        f32.tofile(f)


def read_field(path: str) -> tuple[int, np.ndarray]:
    """Inverse of write_field: (npt, float32 field)."""
    with open(path, "rb") as f:
        npt = int(np.fromfile(f, dtype="int32", count=1)[0])
        f.seek(4)
        return npt, np.fromfile(f, dtype="float32")


def write_model(d: str, nx: int, nz: int, dx: float, dz: float, fields: dict) -> None:
    """A model directory as import_model reads it (fd2d.py:167-182), with the
    x / z coordinate files of a regular nx x nz grid."""
    os.makedirs(d, exist_ok=True)
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    allf = dict(fields)
    allf["x"] = (i * dx).ravel()
    allf["z"] = (j * dz).ravel()
    for k, v in allf.items():
        write_field(os.path.join(d, "proc000000_%s.bin" % k), v, nx * nz)


def read_traces(path: str) -> np.ndarray:
    """Raw float32 trace file (fd2d.py:372)."""
    return np.fromfile(path, dtype="float32")


def write_traces(path: str, traces: np.ndarray) -> None:
    """Raw float32 trace file, receiver-major (fd2d.py:406)."""
    np.asarray(traces, dtype="float32").ravel().tofile(path)
