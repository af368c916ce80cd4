"""Host logic that needs no GPU: sprun-style config inheritance and path
rebasing (scripts/sprun:10-42), and the torch.distributed mpi shim with
world_size 2 over gloo (shot sharding + sums of kernels and misfits)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from seispie_b200.parallel import shard
from seispie_b200.workflow import parse_config


def _write(p, text):
    os.makedirs(os.path.dirname(p), exist_ok=True)
    open(p, "w").write(text)


def test_config_inheritance(tmp_path):
    r = str(tmp_path)
    _write(os.path.join(r, "forward", "config.ini"),
           "[workflow]\nmode = forward\nmpi = no\n[solver]\nmethod = fd2d\nnt = 4800\nsmooth = 1\n"
           "[path]\noutput = output\nmodel_init = model_init\nmodel_true = model_true\ntraces = no\n")
    _write(os.path.join(r, "adjoint", "config.ini"),
           "[workflow]\nmode = adjoint\ninherit = forward\n[solver]\nsmooth = 5\n[path]\noutput = output\n")
    _write(os.path.join(r, "inverse", "config.ini"),
           "[workflow]\nmode = inversion\ninherit = adjoint\n[optimize]\nniter = 10\n[path]\noutput = output\n")
    cfg, wd = parse_config(os.path.join(r, "inverse"), "config.ini")
    assert cfg["workflow"]["mode"] == "inversion"
    assert cfg["solver"]["nt"] == "4800" and cfg["solver"]["smooth"] == "5"
    assert cfg["path"]["output"] == "output"
    # paths inherited from two levels up are rebased twice, 'no' is kept
    assert cfg["path"]["model_init"] == "../adjoint/../forward/model_init"
    assert cfg["path"]["traces"] == "no"
    assert cfg["optimize"]["niter"] == "10"


def test_shards_cover_every_shot_once():
    for n in (1, 5, 32, 64):
        for size in (1, 2, 3, 8):
            got = [i for r in range(size) for i in shard(n, r, size)]
            assert got == list(range(n))


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    from seispie_b200.parallel import TorchMPI
    mpi = TorchMPI(backend="gloo", timeout_s=30)
    try:
        shots = list(shard(7, mpi.rank(), mpi.size()))
        # each shot contributes a kernel and a misfit that identify it
        k = torch.zeros(5, dtype=torch.float64)
        mis = 0.0
        for s in shots:
            k += torch.arange(5, dtype=torch.float64) * (s + 1)
            mis += float(s + 1)
        mpi.allreduce_tensor(k)
        out = np.zeros(1)
        mpi.sum(np.array([mis]), out)
        mpi.sync()
        q.put((rank, shots, k.numpy().tolist(), float(out[0])))
    finally:
        mpi.close()


def test_torch_mpi_shim_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = sum(range(1, 8))
    assert sorted(res[0][1] + res[1][1]) == list(range(7))
    for _, _, k, m in res:
        assert m == total
        assert k == [float(i * total) for i in range(5)]


class _NoStream:
    def synchronize(self):
        pass


def _plugin_rank_main(rank, size, port, nsrc, q):
    """One rank of the plugin's shot sharding: the solver's own _shots,
    _mpi_sum_kernels and _mpi_sum_misfit on CPU kernels."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(size))
    import torch
    from seispie_b200.parallel import TorchMPI
    from seispie_b200.solver.b200 import b200
    mpi = TorchMPI("gloo")
    try:
        s = b200()
        s.nsrc, s.mpi, s.stream = nsrc, mpi, _NoStream()
        shape = (3, 4)
        for name in ("k_lam_f64", "k_mu_f64", "k_rho_f64", "illum_f64", "k_nu_f64", "k_mnc_f64", "k_j_f64"):
            setattr(s, name, torch.zeros(shape, dtype=torch.float64))
        misfit = 0.0
        for shot in s._shots():  # each shot adds a distinct power of two: a double count would show
            for f, k in enumerate(s._summed_fields()):
                k += float(2 ** shot) * (f + 1)
            misfit += float(2 ** shot)
        misfit = s._mpi_sum_misfit(misfit)
        s._mpi_sum_kernels()
        q.put((rank, list(s._shots()), [float(k[0, 0]) for k in s._summed_fields()], misfit))
    finally:
        mpi.close()


def test_plugin_shot_sharding_and_kernel_sum_two_ranks_gloo():
    """Two gloo ranks run the plugin's shot sharding: contiguous shards that
    cover every shot once, and kernels and misfit summed across ranks so
    that every shot counts exactly once (the reference's file exchange,
    solver.py:380-391, added the local kernel twice)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    nsrc = 7
    procs = [ctx.Process(target=_plugin_rank_main, args=(r, 2, port, nsrc, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] + res[1][1] == list(range(nsrc))  # contiguous, disjoint, complete
    total = float(2 ** nsrc - 1)
    for _, _, ks, m in res:
        assert m == total
        assert ks == [total * (f + 1) for f in range(7)]


def test_merge_rule_edges():
    """A section the child lacks comes whole from the parent (paths
    rebased), sections outside the inherited set are not inherited, a
    child's own value wins, 'no' stays 'no'."""
    from seispie_b200.workflow import merge_configs
    parent = {"path": {"model_true": "mt", "traces": "no"}, "solver": {"nt": "10", "dt": "1e-3"},
              "custom": {"x": "1"}}
    child = {"workflow": {"inherit": "p"}, "solver": {"nt": "20"}}
    out = merge_configs(child, parent, "../p")
    assert out["path"] == {"model_true": "../p/mt", "traces": "no"}
    assert out["solver"] == {"nt": "20", "dt": "1e-3"}
    assert "custom" not in out and out["workflow"] == {"inherit": "p"}
