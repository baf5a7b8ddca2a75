"""Loader of liblbm_b200.so (ctypes).  The product path has no CPU fallback:
if the library is missing or a call fails, an exception is raised."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # lbm-cuda_b200/
# LBM_B200_LIB names another build of the library (for instance one compiled
# with different tuning macros); the default is the in-tree build.
LIB_PATH = os.environ.get("LBM_B200_LIB") or os.path.join(PKG_DIR, "liblbm_b200.so")

_P, _I, _F, _D = C.c_void_p, C.c_int, C.c_float, C.c_double
_IP = C.POINTER(C.c_int)

# Argument types of every exported entry point (include/lbm_b200.h).
SIGNATURES = {
    "lbm_core4_step": ([_P] * 6 + [_I, _I, _F, _F, _F, _P], _I),
    "lbm_core4_run": ([_P] * 6 + [_I, _I, _F, _F, _I, _I, _P, _IP], _I),
    "lbm_smemaa_step": ([_P] * 6 + [_I, _I, _F, _F, _I, _P], _I),
    "lbm_blocked_step": ([_P] * 3 + [_I, _I, _F, _F, _I, _P], _I),
    "lbm_macro": ([_P] * 5 + [_I, _I, _F, _P], _I),
    "lbm_visualize": ([_P] * 5 + [_I, _I, _F, _P], _I),
    "lbm_params_default": ([_P, _I, _I], None),
    "lbm_create": ([_P, C.POINTER(C.c_void_p)], _I),
    "lbm_destroy": ([_P], _I),
    "lbm_state_bytes": ([_P], C.c_size_t),
    "lbm_init_equilibrium": ([_P] * 5 + [_P], _I),
    "lbm_run": ([_P] * 4 + [_I, _I, _P, _P, _P, _P, _IP], _I),
    "lbm_run_inplace": ([_P] * 3 + [_I, _P, _P, _P, _P], _I),
    "lbm_run_graph_reset": ([_P], _I),
    "lbm_run_columns": ([_P] * 4 + [_I, _I, _I, _P], _I),
    "lbm_halo_pack": ([_P, _I, _I, _I, _I, _I, _I, _P, _P], _I),
    "lbm_halo_unpack": ([_P, _I, _I, _I, _I, _I, _I, _P, _P], _I),
    "lbm_periodic_halo_x": ([_P, _I, _I, _I, _I, _P], _I),
    "lbm_diag_fp64": ([_P] * 4 + [_P], _I),
    "lbm_forces_fp64": ([_P] * 4 + [_P], _I),
    "lbm_diag_fp64_noalloc": ([_I, _I, _I, _P, _P, _P, _P], _I),
    "lbm_mlp_forward": ([_P, _P, _P, _I, _P], _I),
    "lbm_mlp_forward_act": ([_P, _I, _P, _P, _I, _P], _I),
    "lbm_mlp_grad_act": ([_P, _I, _P, _P, _P, _I, _P, _P, _P, C.c_size_t, _P], _I),
    "lbm_mlp_pack_act": ([_P, _I, _P, _F, _P, _P], _I),
    "lbm_mlp_workspace_bytes": ([_I], C.c_size_t),
    "lbm_mlp_grad": ([_P, _P, _P, _P, _I, _P, _P, _P, C.c_size_t, _P], _I),
    "lbm_mlp_adam": ([_P, _P, _P, _P, _I, _F, _F, _F, _F, _P], _I),
    "lbm_mlp_pack": ([_P, _P, _F, _P, _P], _I),
    "lbm_convert_state": ([_I, _I, _P, _I, _P, _I, _P], _I),
    "lbm_device_error_flags": ([_IP, _I], _I),
    "lbm_selftest_wait_timeout": ([C.c_longlong, _I, _P, _P], _I),
    "lbm_batch_create": ([_P, _P, _I, C.POINTER(C.c_void_p)], _I),
    "lbm_batch_destroy": ([_P], _I),
    "lbm_batch_run": ([_P, _I, _I, _P, _IP], _I),
    "lbm_batch_run_separate": ([_P, _I, _I, _P, _IP], _I),
    "lbm_batch_autotune": ([_P, _P, _IP, _IP], _I),
    "lbm_batch_get_tiles": ([_P, _IP, _IP], _I),
    "lbm_batch_set_tiles": ([_P, _I, _IP], _I),
    "lbm_error_string": ([_I], C.c_char_p),
    "lbm_version": ([], _I),
}


class LbmError(RuntimeError):
    def __init__(self, fn: str, status: int):
        self.status = status
        super().__init__(f"{fn} failed: status {status} ({error_string(status)})")


def build(jobs: int = 8) -> None:
    """Compile liblbm_b200.so in-tree for sm_100a."""
    subprocess.run(["make", "-s", "-C", PKG_DIR, f"-j{jobs}"], check=True)


_lock = threading.Lock()
_lib = None


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                              "(lbm_b200 has no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (argt, rest) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = argt
                fn.restype = rest
            _lib = L
    return _lib


def error_string(status: int) -> str:
    try:
        return lib().lbm_error_string(status).decode()
    except OSError:
        return "?"


def check(fn: str, status: int) -> None:
    if status != 0:
        raise LbmError(fn, status)


def call(name: str, *args) -> int:
    st = getattr(lib(), name)(*args)
    check(name, st)
    return st
