"""Uneven-size multi-instance batches (fwi_multi_run): every instance's
traces are bit-identical to running that instance alone with fwi_run, with
and without CUDA-graph capture, and match the FP64 oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _small_instances():
    from seispie_b200.uneven import make_instances
    return make_instances(6, seed=7, sizes=(40, 90), nts=(60, 220), shots=(2, 4), nrec_per_cell=0.2)


def _alone(inst):
    from seispie_b200.engine import Grid, ShotBatch, build_model, injection_lists, point_ids, ricker_stf
    g = Grid(inst.nx, inst.nz, float(np.float32(inst.h)), float(np.float32(inst.h)))
    m = build_model(inst.mode, g, inst.dt, inst.params, inst.absorb)
    sid = point_ids(inst.src, np.float32(inst.h), np.float32(inst.h), inst.nz)
    rid = point_ids(inst.rec, np.float32(inst.h), np.float32(inst.h), inst.nz)
    b = ShotBatch(m, len(sid), inst.nt, rid)
    stf, _ = ricker_stf(inst.src, inst.nt, inst.dt, "cuda")
    b.clear()
    b.run(b.desc(inj=injection_lists(len(sid), sid, lambda s: s), stf=stf), False, 0, inst.nt)
    return [b.traces(c).cpu().numpy() if b.obs[c] is not None else None for c in range(3)]


def test_uneven_batch_matches_single_runs_bitwise():
    from seispie_b200.uneven import UnevenBatch
    insts = _small_instances()
    assert len({i.nt for i in insts}) > 1 and {i.mode for i in insts} == {"sh", "psv"}
    ub = UnevenBatch(insts)
    ub.prepare()
    ub.clear()
    ub.run()
    torch.cuda.synchronize()
    for k, inst in enumerate(insts):
        ref = _alone(inst)
        got = ub.traces(k)
        for c in range(3):
            if ref[c] is not None:
                assert np.array_equal(got[c].cpu().numpy(), ref[c]), (k, c)
    # the same through one captured graph, replayed twice
    g = ub.capture()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for k, inst in enumerate(insts):
        ref = _alone(inst)
        for c in range(3):
            if ref[c] is not None:
                assert np.array_equal(ub.traces(k)[c].cpu().numpy(), ref[c]), (k, c)


def test_uneven_batch_vs_fp64_oracle():
    from seispie_b200.uneven import UnevenBatch
    from tests.gpu_helpers import oracle_trace_error as oracle_error
    insts = _small_instances()
    ub = UnevenBatch(insts)
    ub.prepare()
    ub.clear()
    ub.run()
    ub.check()
    for k, inst in enumerate(insts):
        assert oracle_error(inst, ub.traces(k), inst.nt) < 1e-5, k
