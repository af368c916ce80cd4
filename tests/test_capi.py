"""The C-ABI library loads on a machine without a GPU, exports every entry
point that include/seispie_b200.h declares, and rejects bad arguments with a
status code and a message before touching the device."""
import ctypes
import subprocess

import pytest

from seispie_b200 import _lib
from seispie_b200._lib import FwiBatch


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.exported_symbols()
    assert len(declared) >= 12
    for name in declared:
        assert hasattr(lib, name), name
    nm = subprocess.run(["nm", "-D", "--defined-only", _lib.lib_path()], capture_output=True, text=True).stdout
    for name in declared:
        assert (" T " + name) in nm, name
    assert lib.fwi_abi_version() == _lib.ABI_VERSION


def test_library_is_built_for_sm100a():
    """Every translation unit was compiled for sm_100a only (the commands
    build.py recorded), and the link used the same target."""
    import json
    import os
    from seispie_b200 import build
    _lib.load()
    assert os.path.exists(build.INFO), "built without build.py's record"
    info = json.load(open(build.INFO))
    assert len(info["compile"]) == len(build.SOURCES)
    for cmd in info["compile"] + [info["link"]]:
        assert "arch=compute_100a,code=sm_100a" in cmd
        assert cmd.count("-gencode") == 1


@pytest.mark.gpu
def test_loaded_device_code_is_sm100():
    """The device code the runtime loaded reports binary version 100."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    assert _lib.load().fwi_binary_version() == 100


def _err():
    buf = ctypes.create_string_buffer(512)
    code = _lib.load().fwi_last_error(buf, 512)
    return code, buf.value.decode()


def _batch(**kw):
    b = FwiBatch()
    b.mode, b.nx, b.nz, b.pitch, b.nshots, b.nt = 0, 16, 16, 16, 1, 10
    b.dx, b.dz, b.dt = 10.0, 10.0, 1e-3
    for k, v in kw.items():
        setattr(b, k, v)
    return b


@pytest.mark.parametrize("kw,msg", [
    (dict(mode=7), "mode"),
    (dict(step_overlap=2), "step_overlap"),
    (dict(pitch=18), "pitch"),
    (dict(pitch=12), "pitch"),
    (dict(nshots=0), "nshots"),
    (dict(nt=0), "nt"),
    (dict(), "sig"),  # no field pointers
])
def test_run_rejects_bad_batches(kw, msg):
    lib = _lib.load()
    rc = lib.fwi_run(ctypes.byref(_batch(**kw)), 0, 0, 1, None)
    assert rc == -1
    code, text = _err()
    assert code == -1 and msg in text


def test_run_rejects_out_of_range_steps():
    lib = _lib.load()
    assert lib.fwi_run(ctypes.byref(_batch()), 0, 5, 6, None) == -1
    assert "steps" in _err()[1]
    assert lib.fwi_run(None, 0, 0, 1, None) == -1


def test_other_entry_points_validate():
    lib = _lib.load()
    assert lib.fwi_smooth(None, 4, None, 4, None, 4, 4, 2, None) == -1
    assert lib.fwi_smooth(8, 4, 8, 4, 8, 4, 4, 0, None) == -1  # sigma 0: the reference divides by it
    assert "sigma" in _err()[1]
    assert lib.fwi_misfit(None, None, None, None, None, 1, 1, 1, 1.0, None) == -1
    assert lib.fwi_vps2lm(None, None, None, 4, None) == -1
    assert lib.fwi_prepare_model(8, None, None, None, 1.0, 4, 8, 8, None, None) == -1
    assert lib.fwi_tile_shape(99, None, None) == -1
    assert lib.fwi_tile_shape(0, None, None) == 0
    assert _lib.tile_shape(0) == (32, 32) and lib.fwi_tile_kind(0) == 2
    assert len(_lib.tile_variants()) >= 3


def test_check_raises_with_message():
    lib = _lib.load()
    with pytest.raises(_lib.FwiError, match="pitch"):
        _lib.check(lib.fwi_run(ctypes.byref(_batch(pitch=18)), 0, 0, 1, None), "fwi_run")


def test_wait_limit_rejects_negative_before_any_cuda_call():
    lib = _lib.load()
    assert lib.fwi_set_wait_limit(-5) == -1
    code, msg = _err()
    assert code == -1 and "polls" in msg

