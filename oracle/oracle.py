"""ctypes binding of the CPU oracle (oracle/lbm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
cpu_baseline leg of bench.py.  Arrays are numpy, C-ordered, populations shaped
(9, H, W), masks (H, W) uint8.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_P = C.c_void_p
_I = C.c_int
_F = C.c_float
_D = C.c_double

_SIGS = {
    "orc_core4_step_f32": [_P, _P, _P, _P, _P, _P, _I, _I, _F, _F, _F, _F],
    "orc_core4_step_f64": [_P, _P, _P, _P, _P, _P, _I, _I, _D, _D, _D, _D],
    "orc_smemaa_launch_f32": [_P, _P, _P, _P, _P, _P, _I, _I, _F, _F, _I],
    "orc_smemaa_launch_f64": [_P, _P, _P, _P, _P, _P, _I, _I, _D, _D, _I],
    "orc_policy_launch_f32": [_P, _P, _P, _I, _I, _F, _F, _I],
    "orc_policy_launch_f64": [_P, _P, _P, _I, _I, _D, _D, _I],
    "orc_macro_f32": [_P, _P, _P, _P, _P, _I, _I, _F],
    "orc_visualize": [_P, _P, _P, _P, _I, _I, _F],
    "orc_general_step_f32": [_P] * 8,
    "orc_general_step_f64": [_P] * 8,
    "orc_num_threads": [],
    "orc_set_threads": [_I],
    "orc_set_mlp": [_P, _P, _D],
}
_RET = {"orc_num_threads": _I}


def build() -> None:
    """Compile the oracle (and, where the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(name: str) -> C.CDLL:
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    for fn, argt in _SIGS.items():
        f = getattr(lib, fn)
        f.argtypes = argt
        f.restype = _RET.get(fn, None)
    return lib


_LIBS: dict = {}


def lib(cpu_baseline: bool = False) -> C.CDLL:
    key = "libcpubase.so" if cpu_baseline else "liboracle.so"
    if key not in _LIBS:
        _LIBS[key] = _load(key)
    return _LIBS[key]


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def _dt(f: np.ndarray) -> str:
    return "f64" if f.dtype == np.float64 else "f32"


def core4_step(mask, f_now, f_out=None, macro=None, tau_inv=1.8, u_in=0.1, cs=0.2, si=1.1, cpu_baseline=False):
    """One lbm_core4.cu step (lbm_core4.cu:7-212); returns (f_out, (ux, uy, rho))."""
    _, H, W = f_now.shape
    f_out = f_now.copy() if f_out is None else f_out
    if macro is None:
        macro = tuple(np.zeros((H, W), dtype=f_now.dtype) for _ in range(3))
    fn = getattr(lib(cpu_baseline), "orc_core4_step_" + _dt(f_now))
    fn(_p(mask), _p(f_now), _p(f_out), _p(macro[0]), _p(macro[1]), _p(macro[2]), W, H, tau_inv, u_in, cs, si)
    return f_out, macro


def core4_run(mask, f0, n_steps, f_b=None, macro=None, **kw):
    """n_steps ping-pong core4 steps starting from f0 (copied); returns (f, (ux, uy, rho))."""
    a = f0.copy()
    b = a.copy() if f_b is None else f_b.copy()
    _, H, W = f0.shape
    if macro is None:
        macro = tuple(np.zeros((H, W), dtype=f0.dtype) for _ in range(3))
    for _ in range(n_steps):
        core4_step(mask, a, b, macro, **kw)
        a, b = b, a
    return a, macro


def smemaa_launch(mask, f_now, f_out=None, macro=None, tau_inv=1.7, u_in=0.1, T=4):
    """One lbm_core_smemaa.cu launch (T BGK steps); returns (f_out, (ux, uy, rho))."""
    _, H, W = f_now.shape
    f_out = f_now.copy() if f_out is None else f_out
    if macro is None:
        macro = tuple(np.zeros((H, W), dtype=f_now.dtype) for _ in range(3))
    fn = getattr(lib(), "orc_smemaa_launch_" + _dt(f_now))
    fn(_p(mask), _p(f_now), _p(f_out), _p(macro[0]), _p(macro[1]), _p(macro[2]), W, H, tau_inv, u_in, T)
    return f_out, macro


def policy_launch(mask, f_now, f_out, tau_inv=1.0, u_in=0.1, T=6):
    """One lbm_core_smemaa_policy.cu launch (T BGK steps) into f_out (updated in place)."""
    _, H, W = f_now.shape
    fn = getattr(lib(), "orc_policy_launch_" + _dt(f_now))
    fn(_p(mask), _p(f_now), _p(f_out), W, H, tau_inv, u_in, T)
    return f_out


def macro(f, mask, macro_in=None, u_in=0.1):
    """lbm_core_smemaa_policy.cu macro_kernel; returns (ux, uy, rho)."""
    _, H, W = f.shape
    out = tuple(np.zeros((H, W), np.float32) for _ in range(3)) if macro_in is None else macro_in
    lib().orc_macro_f32(_p(f), _p(out[0]), _p(out[1]), _p(out[2]), _p(mask), W, H, u_in)
    return out


def visualize(ux, uy, mask, vort_scale=50.0, img=None):
    """visualizekernel (lbm_core4.cu:214-255); returns the (H, W, 4) uint8 image."""
    H, W = ux.shape
    img = np.zeros((H, W, 4), np.uint8) if img is None else img
    lib().orc_visualize(_p(ux), _p(uy), _p(img), _p(mask), W, H, vort_scale)
    return img


BC = {"wall": 0, "periodic": 1, "zouhe": 2, "zouhe_ramp": 3, "outflow": 4}


def set_mlp(params, in_scale, out_scale):
    """Weights of the oracle's learned closure (closure="mlp")."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    sc = np.ascontiguousarray(in_scale, dtype=np.float32)
    lib().orc_set_mlp(_p(p), _p(sc), float(out_scale))


class General:
    """Parameters of the general solver step (lbm_params semantics)."""

    def __init__(self, W, H, collision="mrt", closure="smag", s_nu=1.8, s_e=1.1, s_eps=1.1, s_q=1.1, cs=0.2,
                 bc_left="zouhe_ramp", bc_right="outflow", bc_y="wall", u_in=0.1, u_lid=0.0, ref_clamps=True):
        self.ip = np.array([W, H, 1 if collision == "mrt" else 0, {"none": 0, "smag": 1, "mlp": 2, "mlp_silu": 3}[closure], BC[bc_left],
                            BC[bc_right], BC[bc_y], int(bool(ref_clamps))], dtype=np.int32)
        self.dp = np.array([s_nu, s_e, s_eps, s_q, cs, u_in, u_lid], dtype=np.float64)

    def step(self, mask, f_now, f_out=None, macro=None):
        _, H, W = f_now.shape
        f_out = f_now.copy() if f_out is None else f_out
        if macro is None:
            macro = tuple(np.zeros((H, W), dtype=f_now.dtype) for _ in range(3))
        fn = getattr(lib(), "orc_general_step_" + _dt(f_now))
        fn(_p(self.ip), _p(self.dp), _p(mask), _p(f_now), _p(f_out), _p(macro[0]), _p(macro[1]), _p(macro[2]))
        return f_out, macro

    def run(self, mask, f0, n_steps, macro=None):
        a, b = f0.copy(), f0.copy()
        _, H, W = f0.shape
        if macro is None:
            macro = tuple(np.zeros((H, W), dtype=f0.dtype) for _ in range(3))
        for _ in range(n_steps):
            self.step(mask, a, b, macro)
            a, b = b, a
        return a, macro
