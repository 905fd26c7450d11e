"""ctypes binding of the in-tree C ABI (``include/moraine_b200.h``).

The shared library is built by ``moraine_b200.build`` into ``moraine_b200/lib``. There is
no CPU fallback: if the library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import threading
from ctypes import c_double, c_int, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libmoraine_b200.so"

MR_OK = 0
MR_ERR_INVALID = -1
MR_ERR_CUDA = -2
MR_ERR_UNSUPPORTED = -3
MR_ERR_WORKSPACE = -4

PREC = {"fp32": 0, "bf16": 1, "bf16x3": 2, "fp64": 3, "mixed": 4, "refine": 5}
KS_INPUT = {"intensity": 0, "amplitude": 1}

MAX_NIMAGES = 512
MAX_WINDOW = 4096

P = c_void_p
_SIGNATURES = {
    "mr_last_error": (ctypes.c_char_p, []),
    "mr_abi_version": (c_int, []),
    "mr_kernel_launches": (ctypes.c_uint64, []),
    "mr_set_kernel_timing": (None, [c_int]),
    "mr_kernel_timing": (c_int, [c_int, P, P, P]),
    "mr_gamma_sample_bytes": (c_size_t, [c_int]),
    "mr_set_autotune": (None, [c_int]),
    "mr_set_emi_sub_batch": (c_int, [c_int64]),
    "mr_ks_plan": (c_int, [c_int, c_int, c_int, P, P, P]),
    "mr_ds_chain_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_int, c_int, c_int64]),
    "mr_ds_chain": (c_int, [P, c_int, c_int, c_int, c_int, c_int, c_int, c_double, c_int, c_int, c_int, P, P, P, P,
                            c_int64, P, c_int64, P, c_size_t, P]),
    "mr_ds_chain_async": (c_int, [P, c_int, c_int, c_int, c_int, c_int, c_int, c_double, c_int, c_int, c_int, P, P, P,
                                  P, c_int64, P, c_int64, P, c_size_t, P]),
    "mr_rslc2amp": (c_int, [P, c_int64, P, P]),
    "mr_ras2pc": (c_int, [P, c_int64, c_int64, c_int64, P, c_int64, P, P, P]),
    "mr_pc2ras": (c_int, [P, P, c_int64, c_int64, c_int64, c_int64, P, c_int, P, P, P]),
    "mr_amp_disp": (c_int, [P, c_int64, c_int, P, P]),
    "mr_calamp_workspace_bytes": (c_size_t, []),
    "mr_calamp": (c_int, [P, c_int64, P, P, c_size_t, P]),
    "mr_ad_intf_pc_workspace_bytes": (c_size_t, [c_int, c_int]),
    "mr_ad_intf_pc": (c_int, [P, P, c_int, c_int, P, c_int64, P, c_int, c_int, P, c_int, P, c_size_t, P]),
    "mr_gamma_decode": (c_int, [P, c_int64, c_int, P, c_int64, P]),
    "mr_intensity": (c_int, [P, c_int64, P, P]),
    "mr_ks_workspace_bytes": (c_size_t, [c_int, c_int, c_int]),
    "mr_ks_test": (c_int, [P, c_int, c_int, c_int, c_int, c_int, P, P, c_double, P, P, P, c_size_t, P]),
    "mr_select_shp": (c_int, [P, c_int64, c_int, c_double, P, P, P]),
    "mr_ds_extract_workspace_bytes": (c_size_t, [c_int64]),
    "mr_ds_extract": (c_int, [P, P, c_int, c_int, c_int, c_int, P, P, c_int64, P, P, c_size_t, P]),
    "mr_ds_extract_noalloc": (c_int, [P, P, c_int, c_int, c_int, c_int, P, P, c_int64, P, P]),
    "mr_emperical_co_pc": (c_int, [P, c_int, c_int, c_int, P, c_int64, P, c_int, c_int, c_int, P, c_int, P,
                                   c_int, P]),
    "mr_emperical_co": (c_int, [P, c_int, c_int, c_int, P, c_int, c_int, P, P, P]),
    "mr_uncompress_coh": (c_int, [P, c_int64, c_int, P, c_int, P, P]),
    "mr_emi_workspace_bytes": (c_size_t, [c_int64, c_int]),
    "mr_emi": (c_int, [P, c_int64, c_int, c_int, c_int, P, P, P, P, c_size_t, P]),
    "mr_emi_routed": (c_int, [P, c_int64, c_int, c_int, c_double, P, P, P, P, P, c_size_t, P]),
    "mr_emi_refined": (c_int, [P, c_int64, c_int, c_int, c_double, P, P, P, P, P, c_size_t, P]),
    "mr_ds_temp_coh": (c_int, [P, P, c_int64, c_int, P, c_int, P, P]),
    "mr_temp_coh": (c_int, [P, P, c_int64, c_int, P, c_int, P, P]),
}

_lib = None
_load_lock = threading.Lock()  # serving slots may load the library from several threads


class MoraineError(RuntimeError):
    """A CUDA-side failure reported by the library (status MR_ERR_CUDA)."""


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def load() -> ctypes.CDLL:
    """Load the library (no CUDA context is created by loading)."""
    global _lib
    if _lib is not None:
        return _lib
    with _load_lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"moraine_b200 CUDA library not built ({LIB_PATH}); run `python -m moraine_b200.build`")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        # tune the KS merge tiles on first use of each (device, nimages, window): one stream
        # synchronisation, then the fastest plan; results do not depend on it
        lib.mr_set_autotune(1)
        _lib = lib
        return _lib


def kernel_timing() -> dict:
    """Per-kernel device time recorded since mr_set_kernel_timing(1): name -> (ms, launches)."""
    lib = load()
    name, ms, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_int64()
    out = {}
    for i in range(lib.mr_kernel_timing(-1, None, None, None)):
        lib.mr_kernel_timing(i, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(cnt))
        out[name.value.decode()] = (ms.value, cnt.value)
    return out


def last_error() -> str:
    return load().mr_last_error().decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc == MR_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc == MR_ERR_INVALID:
        raise ValueError(msg)
    if rc == MR_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == MR_ERR_WORKSPACE:
        raise MemoryError(msg)
    raise MoraineError(msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)
