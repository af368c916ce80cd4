"""Failure detection without a GPU fault: a bounded wait that runs out.

Every wait of the library's pipelined kernels is bounded; one that runs out
ends its kernel and sets the device status word, and the product path
checks that word at its sync points and raises.  The test shortens the
poll limit and launches a kernel whose wait can never complete (an mbarrier
nothing arrives at, no copy in flight), so the wait runs out quickly and
harmlessly; then it checks that the engine and the plugin raise, and that
the context is still usable afterwards.
"""
import ctypes

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _status(lib, clear=0):
    v = ctypes.c_int()
    assert lib.fwi_device_status(ctypes.byref(v), clear) == 0
    return v.value


def test_wait_that_runs_out_raises_and_the_context_survives(tmp_path):
    from seispie_b200 import _lib, engine
    from seispie_b200._lib import FwiError, check
    from tests.conftest import load_golden
    from tests.test_gpu_parity import _plugin_case
    lib = _lib.load()
    g = load_golden("sh_grad")
    sol = _plugin_case(tmp_path, g)  # set up (forward runs) with the default limit
    torch.cuda.synchronize()
    _status(lib, clear=1)
    s = engine.stream_handle(None)
    try:
        # only the self-test kernel runs while the limit is short
        check(lib.fwi_set_wait_limit(2000), "fwi_set_wait_limit")
        check(lib.fwi_wait_selftest(s), "fwi_wait_selftest")
        check(lib.fwi_set_wait_limit(0), "fwi_set_wait_limit")
        torch.cuda.synchronize()
        assert _status(lib) == 1
        with pytest.raises(FwiError, match="bounded wait"):
            engine.check_device()
        assert _status(lib) == 0  # the check cleared it
        # the plugin raises at its next sync point when a wait gave up meanwhile
        check(lib.fwi_set_wait_limit(2000), "fwi_set_wait_limit")
        check(lib.fwi_wait_selftest(s), "fwi_wait_selftest")
        check(lib.fwi_set_wait_limit(0), "fwi_set_wait_limit")
        with pytest.raises(FwiError, match="run_kernel"):
            sol.compute_gradient()
    finally:
        lib.fwi_set_wait_limit(0)
        torch.cuda.synchronize()
        _status(lib, clear=1)
    # the context is intact: the same gradient now runs and matches the reference
    from tests.gpu_helpers import rel
    k, misfit, _ = sol.compute_gradient()
    assert rel(k, g["k_mu"]) < 1e-4
    assert _status(lib) == 0
