"""Host-side logic of the b200 plugin that needs no GPU: model file
reading and grid inference, point mapping, injection lists, shot sharding,
and the refusal to start without CUDA."""
import os

import numpy as np
import pytest
import torch

from oracle.oracle import grid_geometry, point_ids
from seispie_b200 import engine
from seispie_b200.io import write_model
from seispie_b200.solver import DeviceArray, b200
from tests.conftest import load_golden


def make_case_dir(tmp_path, g):
    """Directory layout of an adjoint run for the sh_grad golden case."""
    nx, nz = int(g["nx"]), int(g["nz"])
    h = float(g["dx"])
    n = nx * nz
    true = os.path.join(str(tmp_path), "model_true")
    init = os.path.join(str(tmp_path), "model_init")
    write_model(true, nx, nz, h, h, dict(vp=np.full(n, 3000.0), vs=g["true_vs"], rho=np.full(n, 2600.0)))
    write_model(init, nx, nz, h, h, dict(vp=np.full(n, 3000.0), vs=np.full(n, 1732.0), rho=np.full(n, 2600.0)))
    out = os.path.join(str(tmp_path), "output")
    os.makedirs(out, exist_ok=True)
    np.savetxt(os.path.join(str(tmp_path), "src.dat"), g["src"])
    np.savetxt(os.path.join(str(tmp_path), "rec.dat"), g["rec"])
    return dict(model_true=true, model_init=init, sources=os.path.join(str(tmp_path), "src.dat"),
                stations=os.path.join(str(tmp_path), "rec.dat"), output=out)


def test_point_ids_match_reference_geometry():
    g = load_golden("example_geometry")
    s = b200()
    s.nx, s.nz, s.dx, s.dz = int(g["nx"]), int(g["nz"]), g["dx"], g["dz"]
    assert np.array_equal(s._point_ids(g["src"]), g["src_id"])
    assert np.array_equal(s._point_ids(g["rec"]), g["rec_id"])
    with pytest.raises(ValueError):
        s._point_ids(np.array([[-1e9, 0.0]]))


def test_grid_inference():
    """Same answer as the reference's formula where that formula is
    consistent; the right grid where it is not (1024x512, 37x5)."""
    from seispie_b200.solver.b200 import infer_grid
    for nx, nz in ((20, 28), (201, 201), (1024, 512), (37, 5), (512, 1024)):
        i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        x = (i * 7.5).ravel().astype(np.float32)
        z = (j * 7.5).ravel().astype(np.float32)
        gx, gz, dx, dz = infer_grid(x, z, np.int32(nx * nz))
        assert (gx, gz) == (nx, nz) and dx == np.float32(7.5) and dz == np.float32(7.5)
        rx, rz, rdx, rdz = grid_geometry(x, z, np.int32(nx * nz))
        if rx * rz == nx * nz:
            assert (rx, rz, rdx, rdz) == (gx, gz, dx, dz)
    # the reference formula itself mis-infers 1024x512
    i, j = np.meshgrid(np.arange(1024), np.arange(512), indexing="ij")
    assert grid_geometry((i * 10.0).ravel().astype(np.float32), (j * 10.0).ravel().astype(np.float32),
                         np.int32(1024 * 512))[0] == 1025


def test_injection_lists():
    ptr, cell, row = engine.injection_lists(3, np.array([5, 9, 13]), lambda s: s)
    assert list(ptr) == [0, 1, 2, 3] and list(cell) == [5, 9, 13] and list(row) == [0, 1, 2]
    ptr, cell, row = engine.injection_lists(2, np.array([5, 9]), lambda s: -1)
    assert list(ptr) == [0, 2, 4] and list(cell) == [5, 9, 5, 9] and list(row) == [0, 1, 0, 1]
    ptr, cell, row = engine.adjoint_injection_lists(2, np.array([3, 4, 7]))
    assert list(ptr) == [0, 3, 6] and list(cell) == [3, 4, 7, 3, 4, 7] and list(row) == list(range(6))


def test_pitch():
    assert [engine.pitch_for(n) for n in (1, 4, 5, 201, 512)] == [4, 4, 8, 204, 512]


class FakeMPI:
    def __init__(self, rank, size):
        self._r, self._s = rank, size

    def rank(self):
        return self._r

    def size(self):
        return self._s


def test_shot_sharding_covers_every_shot_once():
    for nsrc in (1, 7, 12, 64):
        for size in (1, 2, 3, 8):
            seen = []
            for r in range(size):
                s = b200()
                s.nsrc, s.mpi = nsrc, FakeMPI(r, size)
                seen += s._shots()
            assert sorted(seen) == list(range(nsrc))


def test_device_array_copy_to_host():
    t = torch.arange(12, dtype=torch.float32).view(3, 4)
    a = DeviceArray(t, nz=3)
    out = np.zeros(9, np.float32)
    a.copy_to_host(out)
    assert list(out) == [0, 1, 2, 4, 5, 6, 8, 9, 10]
    assert a.size == 9


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU refusal")
def test_setup_refuses_without_cuda():
    s = b200()
    s.config = dict(nt="10", dt="1e-3", sh="yes", psv="no")
    s.path, s.mpi = {}, None
    with pytest.raises(RuntimeError, match="CUDA"):
        s.setup(None)


def test_exact_adjoint_fixed_bytes():
    """The memory bound the plugin sizes its stored tail against: checkpoints
    every K steps over all nt steps, K steps of per-step stores, two copies
    of the state and the traces, all of nshots shots."""
    from seispie_b200._lib import FWI_PSV, FWI_SPIN
    from seispie_b200.adjoint import default_segment, fixed_bytes
    from seispie_b200.engine import Grid
    g = Grid(1024, 510, 10.0, 10.0)  # pitch 512
    field = 4 * 64 * 1024 * 512
    # displacement-free P-SV: a checkpoint is 3 stress + 2 velocity fields, a step stores
    # 3 strain terms and 2 divergences, so K = sqrt(nt)
    k = default_segment(6000, FWI_PSV, 64, g)
    assert k == 77
    # 78 checkpoints, 77 steps of stores, forward and adjoint batches of 2 x (3 + 2) fields,
    # and 2 components x (traces, data, trace gradients)
    want = (78 * 5 + 77 * 5 + 2 * 10) * field + 3 * 4 * 64 * 256 * 6000 * 2
    assert fixed_bytes(6000, FWI_PSV, 64, g, 256) == want
    # the overlapped backward holds a second segment of stores, so K = sqrt(nt / 2) = 55
    assert default_segment(6000, FWI_PSV, 64, g, overlap=True) == 55
    assert fixed_bytes(6000, FWI_PSV, 64, g, 256, overlap=True) == \
        (110 * 5 + 2 * 55 * 5 + 2 * 10) * field + 3 * 4 * 64 * 256 * 6000 * 2
    # no density kernel: a step stores the 3 strain terms only, K = sqrt(5 nt / 3) = 100
    assert default_segment(6000, FWI_PSV, 64, g, density=False) == 100
    assert fixed_bytes(6000, FWI_PSV, 64, g, 256, density=False) == \
        (60 * 5 + 100 * 3 + 2 * 10) * field + 3 * 4 * 64 * 256 * 6000 * 2
    # an explicit segment; the spin state is 6 stress + 2 x 3 velocity/displacement fields,
    # a step stores 6 strain terms and 3 divergences, a batch holds 2 x (6 + 3) + 3 fields
    assert fixed_bytes(100, FWI_SPIN, 2, Grid(8, 8, 1.0, 1.0), 0, segment=10) == \
        (10 * 12 + 10 * 9 + 2 * 21) * 4 * 2 * 8 * 8


def test_max_tail_bytes_is_the_longest_tail_that_fits():
    """The stored tail is sized so that checkpoints (of the steps before it),
    one segment of stores, the tail, both batches and the traces fit the
    budget, and one more tail step would not."""
    import math
    from seispie_b200._lib import FWI_PSV
    from seispie_b200.adjoint import default_segment, max_tail_bytes
    from seispie_b200.engine import Grid
    g = Grid(512, 510, 10.0, 10.0)  # pitch 512
    nt, ns, nrec = 4000, 32, 256
    field = 4 * ns * 512 * 512
    k1 = default_segment(nt, FWI_PSV, ns, g)
    k2 = default_segment(nt, FWI_PSV, ns, g, overlap=True)

    def need(t, segs=1):
        k = k2 if segs == 2 else k1
        return (math.ceil((nt - t) / k) * 5 + segs * k * 5 + t * 5 + 20) * field + 3 * 4 * ns * nrec * nt * 2

    for budget in (30e9, 100e9, 160e9):
        t = max_tail_bytes(nt, FWI_PSV, ns, g, budget, nrec) // (5 * field)
        assert 0 < t < nt and need(t) <= budget < need(t + 1)
        t2 = max_tail_bytes(nt, FWI_PSV, ns, g, budget, nrec, overlap=True) // (5 * field)
        if need(0, 2) <= budget:
            assert 0 < t2 < t and need(t2, 2) <= budget < need(t2 + 1, 2)
        else:  # not even the tail-free overlapped backward fits: no tail
            assert t2 == 0
    assert max_tail_bytes(nt, FWI_PSV, ns, g, 1e9, nrec) == 0  # nothing fits: no tail
    assert max_tail_bytes(100, FWI_PSV, 1, Grid(8, 8, 1.0, 1.0), 1e12, 0) == 100 * 5 * 4 * 8 * 8


def test_gradient_graph_key():
    """The kept gradient graph is reused only while the shots, the model's
    and time functions' device buffers and the step settings are the same;
    no graph with cuda_graph = no or a batch-memory cap."""
    from types import SimpleNamespace
    s = b200()
    s.config = dict(combine_sources="no")
    s.batch_memory, s.nt, s.dt, s.tile, s.kernel_rho = 0.0, 100, 1e-3, 0, False
    t = lambda: torch.zeros(4)  # noqa: E731
    s.model = SimpleNamespace(rho=t(), lam=t(), mu=t(), bound=t(), buo=t())
    s.stf_x, s.stf_y, s.stf_z = t(), t(), t()
    s.src_id, s.rec_id = np.array([3, 7], np.int32), np.array([1, 2, 5], np.int32)
    k = s._graph_key(1, [0, 1])
    assert k is not None and k == s._graph_key(1, [0, 1])
    assert s._graph_key(1, [1]) != k  # other shots
    s.model.mu.add_(1.0)  # values change in place: same buffers, same graph
    assert s._graph_key(1, [0, 1]) == k
    s.model.mu = t()  # a new buffer
    assert s._graph_key(1, [0, 1]) != k
    k = s._graph_key(1, [0, 1])
    s.kernel_rho = True
    assert s._graph_key(1, [0, 1]) != k
    s.kernel_rho = False
    s.rec_id = np.array([1, 2, 6], np.int32)
    assert s._graph_key(1, [0, 1]) != k
    s.batch_memory = 2.0 ** 30
    assert s._graph_key(1, [0, 1]) is None
    s.batch_memory = 0.0
    s.config["cuda_graph"] = "no"
    assert s._graph_key(1, [0, 1]) is None
    s._graphs = {("x",): object()}
    s._drop_graphs()
    assert s._graphs == {}
