"""ctypes bindings: libsus2sh.so (the engine: include/sus2sh.h and its
diagnostics include/sus2sh_diag.h) and libsus2sh_tools.so (model writer,
structure and integrator helpers, FMA probe: include/sus2sh_tools.h).  There
is no fallback: if a CUDA library is missing, loading it raises."""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libsus2sh.so")
TOOLS_PATH = os.path.join(PKG_DIR, "libsus2sh_tools.so")

# Every symbol the public headers declare (checked by the CPU test suite).
EXPORTS = (
    "sus2sh_is_sus2_sh_file", "sus2sh_create", "sus2sh_compute", "sus2sh_destroy",
    "sus2sh_cutoff", "sus2sh_last_error", "sus2sh_sync", "sus2sh_forward", "sus2sh_backward",
    "sus2sh_compute_host", "sus2sh_model_info", "sus2sh_profile", "sus2sh_profile_read",
    "sus2sh_cg_energy_noalloc", "sus2sh_param_grad", "sus2sh_compute_batch", "sus2sh_param_grad_batch",
    "sus2sh_cg_kernel_info", "sus2sh_zbl_pair", "sus2sh_real_sh", "sus2sh_edge_kernel_info",
    "sus2sh_model_edge_kernel_info", "sus2sh_batch_kernel_info",
)
TOOLS_EXPORTS = (
    "sus2sh_tools_last_error", "sus2sh_write_synthetic_model", "sus2sh_standard_graph_counts",
    "sus2sh_md_kick_drift", "sus2sh_md_kick", "sus2sh_reduce", "sus2sh_random_insertion",
    "sus2sh_measure_fma_peak",
)

_lib = None
_tools = None


class EngineError(RuntimeError):
    pass


def load() -> ctypes.CDLL:
    """Loads the engine library once and declares the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineError(f"libsus2sh.so not built ({LIB_PATH}); run `make -C gpumd-sus2-sh_b200`")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    sig = {
        "sus2sh_is_sus2_sh_file": (I, [S]),
        "sus2sh_create": (I, [S, I, I, P, P]),
        "sus2sh_compute": (I, [P, I, P, P, P, P, P, P, P, P]),
        "sus2sh_destroy": (None, [P]),
        "sus2sh_cutoff": (D, [P]),
        "sus2sh_last_error": (S, []),
        "sus2sh_sync": (I, [P, P]),
        "sus2sh_forward": (I, [P, I, P, P, P, P, P, P]),
        "sus2sh_backward": (I, [P, P, P, P, P]),
        "sus2sh_compute_host": (I, [P, I, P, P, P, P, P, P, P, P]),
        "sus2sh_model_info": (I, [P, P, I]),
        "sus2sh_profile": (I, [P, I]),
        "sus2sh_cg_energy_noalloc": (I, [P, I, P, P, P, P, P]),
        "sus2sh_param_grad": (I, [P, I, P, P, P, P, P, P, P, P, P]),
        "sus2sh_compute_batch": (I, [P, I, I, P, P, P, P, P, P, P, P, P, P, P]),
        "sus2sh_param_grad_batch": (I, [P, I, I, P, P, P, P, P, P, P, P, P, P]),
        "sus2sh_profile_read": (I, [P, P, I]),
        "sus2sh_cg_kernel_info": (I, [S, I, I, P, P, ctypes.c_size_t]),
        "sus2sh_zbl_pair": (I, [I, I, D, D, D, P, P]),
        "sus2sh_real_sh": (I, [I, D, D, D, P, P, P]),
        "sus2sh_edge_kernel_info": (I, [I, I, I, I, P, P, P, ctypes.c_char_p, ctypes.c_size_t]),
        "sus2sh_model_edge_kernel_info": (I, [S, P, ctypes.c_char_p, ctypes.c_size_t]),
        "sus2sh_batch_kernel_info": (I, [S, P, ctypes.c_char_p, ctypes.c_size_t]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def load_tools() -> ctypes.CDLL:
    """Loads libsus2sh_tools.so once (it links libsus2sh.so)."""
    global _tools
    if _tools is not None:
        return _tools
    if not os.path.exists(TOOLS_PATH):
        raise EngineError(f"libsus2sh_tools.so not built ({TOOLS_PATH}); run `make -C gpumd-sus2-sh_b200`")
    lib = ctypes.CDLL(TOOLS_PATH)
    P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    sig = {
        "sus2sh_tools_last_error": (S, []),
        "sus2sh_write_synthetic_model": (I, [S, I, I, I, I, P, I, I, D, D, I, P, D, D, D, D,
                                             ctypes.c_ulonglong]),
        "sus2sh_standard_graph_counts": (I, [I, I, I, P, I, P]),
        "sus2sh_md_kick_drift": (I, [I, D, P, P, P, P, P, P, P, P]),
        "sus2sh_md_kick": (I, [I, D, P, P, P, P, P]),
        "sus2sh_reduce": (I, [I, P, P, P, P]),
        "sus2sh_random_insertion": (I, [I, D, D, D, D, ctypes.c_ulonglong, P]),
        "sus2sh_measure_fma_peak": (I, [I, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _tools = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().sus2sh_last_error()
        raise EngineError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


def check_tools(rc: int, what: str) -> None:
    if rc != 0:
        msg = load_tools().sus2sh_tools_last_error()
        raise EngineError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")
