"""Host logic of bench.py's multi-GPU modes (no GPU): every shot of the job
is owned by exactly one rank, weak scaling grows the survey with the ranks
and --shard splits a fixed survey, and the JSON config counts the cell
updates of the whole job."""
import argparse
import sys

import pytest

sys.path.insert(0, ".")


def _args(**kw):
    a = dict(shots=32, nx=512, nz=512, nrec=256, nt=4000, sae=10, sigma=4, shard=False, gradient="exact")
    a.update(kw)
    return argparse.Namespace(**a)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
@pytest.mark.parametrize("shard", [False, True])
def test_shots_partitioned_once(world, shard):
    import bench
    from seispie_b200.parallel import shard as block
    a = _args(shard=shard)
    ntot = bench.total_shots(a, world)
    assert ntot == (32 if shard else 32 * world)
    owned = [s for r in range(world) for s in block(ntot, r, world)]
    assert owned == list(range(ntot))  # contiguous blocks in rank order, each shot once
    sizes = [len(block(ntot, r, world)) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


def test_config_counts_the_whole_job():
    import bench
    a = _args()
    w = bench.workload(a)
    c1 = bench.config_of(a, w, world=1)
    c8 = bench.config_of(a, w, world=8)
    assert c1["cells_per_step"] == 2 * 32 * 512 * 512 * 4000
    assert c8["shots"] == 256 and c8["shots_per_rank"] == 32
    assert c8["cells_per_step"] == 8 * c1["cells_per_step"]
    cs = bench.config_of(_args(shard=True), w, world=8)
    assert cs["shots"] == 32 and cs["shots_per_rank"] == 4 and cs["cells_per_step"] == c1["cells_per_step"]


def test_config_names_the_launch_modes():
    """The line says whether the value comes from the graph-replayed
    gradient and whether the steps launch early; the CPU reference arm uses
    neither."""
    import bench
    w = bench.workload(_args())
    c = bench.config_of(_args(impl="b200", graph=1, step_overlap=1), w)
    assert c["cuda_graph"] is True and c["step_overlap"] is True
    c = bench.config_of(_args(impl="b200", graph=0, step_overlap=0), w)
    assert c["cuda_graph"] is False and c["step_overlap"] is False
    c = bench.config_of(_args(impl="b200", graph=1, gradient="reference"), w)
    assert c["cuda_graph"] is False  # the continuous-adjoint path is launched step by step
    c = bench.config_of(_args(impl="reference", graph=1, step_overlap=1), w)
    assert c["cuda_graph"] is False and c["step_overlap"] is False
