"""The C-ABI library loads without a GPU and exports every entry point that
include/lbm_b200.h declares (no compute calls here)."""
import ctypes as C
import os
import re

import lbm_b200 as L
from lbm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "lbm_core4_step" in names and "lbm_smemaa_step" in names and "lbm_blocked_step" in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_cpu_only_calls():
    lib = L.lib()
    assert lib.lbm_version() >= 100
    assert lib.lbm_error_string(1001) == b"invalid argument"
    # argument validation happens before any CUDA call
    assert lib.lbm_core4_step(None, None, None, None, None, None, 8, 8, 1.0, 0.1, 1.0, None) == 1001
    assert lib.lbm_smemaa_step(C.c_void_p(16), C.c_void_p(16), C.c_void_p(32), C.c_void_p(16), C.c_void_p(16),
                               C.c_void_p(16), 64, 64, 1.0, 0.1, 3, None) == 1002  # odd T


def test_params_default_match_reference_constants():
    from lbm_b200.solver import default_params

    p = default_params(2048, 512)
    assert (p.W, p.H) == (2048, 512)
    assert abs(p.s_e - 1.1) < 1e-7 and abs(p.cs_smag - 0.2) < 1e-7  # lbm_core4.cu:6,123
    assert abs(p.s_nu - 1.8) < 1e-6 and abs(p.u_in - 0.1) < 1e-7  # lbm_mine2.py:77-78
