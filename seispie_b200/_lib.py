"""ctypes binding of libseispie_b200.so (include/seispie_b200.h).

The library is loaded from seispie_b200/_build/.  There is no fallback: if it
is missing or CUDA is unavailable the import of the solver fails with an
error that says so.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

FWI_SH, FWI_PSV, FWI_SPIN = 0, 1, 2
MODES = {"sh": FWI_SH, "psv": FWI_PSV, "spin": FWI_SPIN}
ABI_VERSION = 7

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class FwiBatch(ctypes.Structure):
    """Mirror of struct fwi_batch (include/seispie_b200.h)."""
    _fields_ = [
        ("mode", ctypes.c_int), ("nx", ctypes.c_int), ("nz", ctypes.c_int), ("pitch", ctypes.c_int),
        ("nshots", ctypes.c_int), ("nt", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
        ("dt", ctypes.c_double), ("cur", ctypes.c_int), ("tile", ctypes.c_int),
        ("sig", (_vp * 6) * 2), ("vel", (_vp * 3) * 2), ("disp", _vp * 3),
        ("buo", _vp), ("buo_j", _vp), ("bound", _vp), ("lam", _vp), ("mu", _vp), ("nu", _vp), ("mnc", _vp),
        ("inj_ptr", _vp), ("inj_cell", _vp), ("inj_row", _vp), ("stf", _vp * 3),
        ("nrec", ctypes.c_int), ("rec_cell", _vp), ("obs", _vp * 3),
        ("sae", ctypes.c_int), ("nsa", ctypes.c_int), ("snap_u", _vp * 3), ("snap_v", _vp * 3),
        ("k_lam", _vp), ("k_mu", _vp), ("k_rho", _vp),
        ("seg_e", _vp * 6), ("seg_ds", _vp * 3), ("seg0", ctypes.c_int), ("nseg", ctypes.c_int),
        ("k_nu", _vp), ("k_mnc", _vp), ("k_buoj", _vp), ("rec_order", _vp),
        ("ring", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("adj_tile", ctypes.c_int),
        ("step_overlap", ctypes.c_int),
    ]


class FwiError(RuntimeError):
    """A non-zero status from libseispie_b200."""


_LIB = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load (building first, if needed and allowed) the CUDA library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise ImportError("libseispie_b200.so not built (run python -m seispie_b200.build)")
        _build.build()
    lib = ctypes.CDLL(path)
    sigs = {
        "fwi_abi_version": ([], ctypes.c_int),
        "fwi_launch_count": ([], ctypes.c_longlong),
        "fwi_binary_version": ([], ctypes.c_int),
        "fwi_last_error": ([ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "fwi_device_status": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
        "fwi_set_wait_limit": ([ctypes.c_int], ctypes.c_int),
        "fwi_wait_selftest": ([_vp], ctypes.c_int),
        "fwi_unet_conv_path": ([ctypes.c_int], ctypes.c_int),
        "fwi_tile_shape": ([ctypes.c_int, _ip, _ip], ctypes.c_int),
        "fwi_tile_kind": ([ctypes.c_int], ctypes.c_int),
        "fwi_vps2lm": ([_vp, _vp, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
        "fwi_lm2vps": ([_vp, _vp, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
        "fwi_set_bound": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_ricker": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp, _vp, _vp, _vp], ctypes.c_int),
        "fwi_prepare_model": ([_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_longlong, _vp, _vp, _vp, _vp],
                              ctypes.c_int),
        "fwi_run": ([ctypes.POINTER(FwiBatch), ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_run_transposed": ([ctypes.POINTER(FwiBatch), ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_multi_workspace_bytes": ([ctypes.c_int], ctypes.c_longlong),
        "fwi_multi_prepare": ([ctypes.POINTER(ctypes.POINTER(FwiBatch)), ctypes.c_int, _vp], ctypes.c_int),
        "fwi_multi_run": ([ctypes.POINTER(ctypes.POINTER(FwiBatch)), ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                           _vp], ctypes.c_int),
        "fwi_misfit": ([_vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp],
                       ctypes.c_int),
        "fwi_misfit_partials": ([ctypes.c_int, ctypes.c_int], ctypes.c_longlong),
        "fwi_reduce_partials": ([], ctypes.c_longlong),
        "fwi_misfit_tracegrad": ([_vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  _vp], ctypes.c_int),
        "fwi_trace_suffix_sum": ([_vp, _vp, ctypes.c_longlong, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_energy_accumulate": ([_vp, ctypes.c_int, ctypes.c_longlong, _vp, _vp], ctypes.c_int),
        "fwi_dot": ([_vp, _vp, ctypes.c_longlong, _vp, _vp, _vp], ctypes.c_int),
        "fwi_absmax": ([_vp, ctypes.c_longlong, _vp, _vp, _vp], ctypes.c_int),
        "fwi_axpby": ([_vp, ctypes.c_double, _vp, ctypes.c_double, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
        "fwi_misfit_noalloc": ([_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp],
                               ctypes.c_int),
        "fwi_smooth": ([_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp],
                       ctypes.c_int),
        "fwi_unet_conv3x3": ([_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_unet_flip_weights": ([_vp, _vp, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_unet_relu_bwd": ([_vp, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
        "fwi_unet_wgrad_partials": ([ctypes.c_int] * 5, ctypes.c_longlong),
        "fwi_unet_conv3x3_wgrad": ([_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, _vp, _vp, _vp, _vp], ctypes.c_int),
        "fwi_unet_pool2": ([_vp, _vp] + [ctypes.c_int] * 4 + [_vp], ctypes.c_int),
        "fwi_unet_pool2_bwd": ([_vp, _vp] + [ctypes.c_int] * 5 + [_vp], ctypes.c_int),
        "fwi_unet_up2": ([_vp, _vp] + [ctypes.c_int] * 4 + [_vp], ctypes.c_int),
        "fwi_unet_up2_bwd": ([_vp, _vp] + [ctypes.c_int] * 4 + [_vp], ctypes.c_int),
        "fwi_unet_head": ([_vp, _vp, _vp, _vp] + [ctypes.c_int] * 3 + [_vp], ctypes.c_int),
        "fwi_unet_head_bwd": ([_vp] * 6 + [ctypes.c_int] * 3 + [_vp], ctypes.c_int),
        "fwi_unet_pack": ([_vp, _vp] + [ctypes.c_int] * 3 + [_vp], ctypes.c_int),
        "fwi_unet_adam": ([_vp, _vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                           ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp], ctypes.c_int),
        "fwi_unet_mse_partials": ([], ctypes.c_longlong),
        "fwi_unet_mse": ([_vp, _vp, _vp, _vp, _vp, ctypes.c_longlong, _vp], ctypes.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.fwi_abi_version() != ABI_VERSION:
        raise ImportError("libseispie_b200.so ABI %d, expected %d" % (lib.fwi_abi_version(), ABI_VERSION))
    _LIB = lib
    return lib


def exported_symbols():
    """Names declared in include/seispie_b200.h (used by the ABI test)."""
    import re
    hdr = os.path.join(os.path.dirname(_build.PKG), "include", "seispie_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char \*)\s+\**(fwi_\w+)\s*\(", text, re.M)))


def tile_variants() -> list[int]:
    """Step-kernel tile variants the library offers (1.. ; 0 aliases the default)."""
    lib = load()
    out, t = [], 1
    x, z = ctypes.c_int(), ctypes.c_int()
    while lib.fwi_tile_shape(t, ctypes.byref(x), ctypes.byref(z)) == 0:
        out.append(t)
        t += 1
    return out


def tile_shape(tile: int) -> tuple[int, int]:
    x, z = ctypes.c_int(), ctypes.c_int()
    check(load().fwi_tile_shape(tile, ctypes.byref(x), ctypes.byref(z)), "fwi_tile_shape")
    return x.value, z.value


def tile_label(tile: int) -> str:
    """e.g. '9:32x32/tma' -- variant id, interior tile and staging kind."""
    tx, tz = tile_shape(tile)
    kind = {0: "generic", 1: "rw", 2: "tma"}[load().fwi_tile_kind(tile)]
    return "%d:%dx%d/%s" % (tile, tx, tz, kind)


def check(rc: int, what: str = "") -> None:
    """Raise FwiError with the library's message for a non-zero status."""
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        load().fwi_last_error(buf, 512)
        raise FwiError("%s failed (%d): %s" % (what or "libseispie_b200", rc, buf.value.decode()))


def ptr(t) -> int | None:
    """Device address of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()
