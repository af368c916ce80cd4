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
