"""lbm_b200: B200-native D2Q9 lattice-Boltzmann collide-stream library.

Python host side of liblbm_b200.so:

* :class:`RefCompatModule` mirrors the reference drivers' kernel handles
  (``cp.RawModule(...).get_function(name)`` then ``kern(grid, block, args)``,
  lbm_mine2.py:69-80), so a driver swaps one line to use this library;
* thin wrappers of the C entry points taking torch (or cupy) device arrays.

All work is enqueued on the caller's current stream; nothing synchronises.
"""
from __future__ import annotations

import ctypes as C

from . import init  # noqa: F401
from ._lib import LbmError, build, call, lib  # noqa: F401

__all__ = ["RefCompatModule", "LbmError", "build", "lib", "init", "core4_step", "core4_run", "smemaa_step",
           "blocked_step", "macro", "visualize"]


def _ptr(a) -> C.c_void_p:
    """Device pointer of a torch tensor, a cupy array or a raw integer."""
    if a is None:
        return C.c_void_p(0)
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):  # torch
        return C.c_void_p(a.data_ptr())
    data = getattr(a, "data", None)
    if data is not None and hasattr(data, "ptr"):  # cupy
        return C.c_void_p(data.ptr)
    raise TypeError(f"cannot take a device pointer of {type(a)!r}")


def _array_library(arrays) -> str | None:
    """"torch" or "cupy" for the first device array among `arrays`, else None."""
    for a in arrays:
        if a is None or isinstance(a, int):
            continue
        if hasattr(a, "data_ptr"):
            return "torch"
        data = getattr(a, "data", None)
        if data is not None and hasattr(data, "ptr"):
            return "cupy"
    return None


def _torch_stream():
    try:
        import torch
    except ImportError:
        return None
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return None


def _cupy_stream():
    try:
        import cupy  # type: ignore
    except ImportError:
        return None
    return C.c_void_p(cupy.cuda.get_current_stream().ptr)


def _stream(stream=None, *arrays) -> C.c_void_p:
    """The stream to launch on: explicit; else the current stream of the array
    library the arguments come from (cupy arrays: cupy's, so that a driver
    capturing a graph on a cupy stream, lbm_mine2.py:75-81, captures these
    launches too, even in a process that has also initialised torch; torch
    tensors: torch's); else torch's current stream when torch is initialised,
    else cupy's, else the legacy default stream."""
    if stream is not None:
        if isinstance(stream, int):
            return C.c_void_p(stream)
        for attr in ("cuda_stream", "ptr"):
            if hasattr(stream, attr):
                return C.c_void_p(getattr(stream, attr))
        raise TypeError(f"unknown stream object {type(stream)!r}")
    kind = _array_library(arrays)
    order = (_cupy_stream, _torch_stream) if kind == "cupy" else (_torch_stream, _cupy_stream)
    for pick in order:
        s = pick()
        if s is not None:
            return s
    return C.c_void_p(0)


def core4_step(mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in, tau_inv_bnd=None, stream=None):
    """lbm_core4_step: one MRT+Smagorinsky step (lbm_core4.cu:7-212)."""
    tb = tau_inv if tau_inv_bnd is None else tau_inv_bnd
    call("lbm_core4_step", _ptr(mask), _ptr(f_now), _ptr(f_out), _ptr(ux), _ptr(uy), _ptr(rho), int(W), int(H),
         float(tau_inv), float(u_in), float(tb), _stream(stream, f_now))


def core4_run(mask, f_a, f_b, ux, uy, rho, W, H, tau_inv, u_in, n_steps, T=4, stream=None) -> int:
    """n_steps core4 steps fused T per launch; returns 1 if the result is in f_b, else 0."""
    out = C.c_int(0)
    call("lbm_core4_run", _ptr(mask), _ptr(f_a), _ptr(f_b), _ptr(ux), _ptr(uy), _ptr(rho), int(W), int(H),
         float(tau_inv), float(u_in), int(n_steps), int(T), _stream(stream, f_a), C.byref(out))
    return out.value


def smemaa_step(mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in, T=4, stream=None):
    """lbm_smemaa_step: T BGK steps, shared-memory AA pattern (lbm_core_smemaa.cu:12-547)."""
    call("lbm_smemaa_step", _ptr(mask), _ptr(f_now), _ptr(f_out), _ptr(ux), _ptr(uy), _ptr(rho), int(W), int(H),
         float(tau_inv), float(u_in), int(T), _stream(stream, f_now))


def blocked_step(mask, f_now, f_out, W, H, tau_inv, u_in, T=6, stream=None):
    """lbm_blocked_step: T BGK steps, end-fused (lbm_core_smemaa_policy.cu:78-425)."""
    call("lbm_blocked_step", _ptr(mask), _ptr(f_now), _ptr(f_out), int(W), int(H), float(tau_inv), float(u_in),
         int(T), _stream(stream, f_now))


def macro(f, ux, uy, rho, mask, W, H, u_in, stream=None):
    """lbm_macro: u, v, rho from canonical f (lbm_core_smemaa_policy.cu:431-476)."""
    call("lbm_macro", _ptr(f), _ptr(ux), _ptr(uy), _ptr(rho), _ptr(mask), int(W), int(H), float(u_in),
         _stream(stream, f))


def visualize(ux, uy, rho, image, mask, W, H, vort_scale, stream=None):
    """lbm_visualize: vorticity colour map into an RGBA8 device buffer (lbm_core4.cu:214-255)."""
    call("lbm_visualize", _ptr(ux), _ptr(uy), _ptr(rho), _ptr(image), _ptr(mask), int(W), int(H),
         float(vort_scale), _stream(stream, ux))


class _Kernel:
    def __init__(self, fn, name):
        self._fn = fn
        self.name = name

    def __call__(self, grid, block, args, stream=None, **_):
        """Reference call shape ``kern(grid, block, args)``; grid and block are ignored
        (this library picks its own launch shape)."""
        return self._fn(*args, stream=stream)


class RefCompatModule:
    """Drop-in for ``cp.RawModule(code=<reference .cu>)`` in the reference drivers.

    ``kind`` names the reference source: ``"core4"`` (lbm_core4.cu), ``"smemaa"``
    (lbm_core_smemaa.cu, T=4), ``"policy"`` / ``"endfused"``
    (lbm_core_smemaa_policy.cu / lbm_core_smemaa_endfused.cu, T=6).
    ``get_function`` returns callables with the reference's positional
    arguments (lbm_core4.cu:7-13, lbm_core_smemaa.cu:12-15,
    lbm_core_smemaa_policy.cu:78-80 and :431-433, visualizekernel)."""

    _T = {"core4": 1, "smemaa": 4, "policy": 6, "endfused": 6}

    def __init__(self, kind: str = "core4", T: int | None = None):
        if kind not in self._T:
            raise ValueError(f"unknown reference kernel family {kind!r}")
        self.kind = kind
        self.T = self._T[kind] if T is None else int(T)
        lib()  # fail loudly now if the library is missing

    def get_function(self, name: str) -> _Kernel:
        k = self.kind
        if name == "visualizekernel":
            return _Kernel(lambda ux, uy, rho, image, mask, W, H, vs, stream=None:
                           visualize(ux, uy, rho, image, mask, W, H, vs, stream), name)
        if name == "fused_lbmkernel":
            if k == "core4":
                return _Kernel(lambda mask, fn, fo, ux, uy, rho, W, H, ti, u, tb, stream=None:
                               core4_step(mask, fn, fo, ux, uy, rho, W, H, ti, u, tb, stream), name)
            if k == "smemaa":
                return _Kernel(lambda mask, fn, fo, ux, uy, rho, W, H, ti, u, stream=None:
                               smemaa_step(mask, fn, fo, ux, uy, rho, W, H, ti, u, self.T, stream), name)
            return _Kernel(lambda mask, fn, fo, W, H, ti, u, stream=None:
                           blocked_step(mask, fn, fo, W, H, ti, u, self.T, stream), name)
        if name == "macro_kernel" and k in ("policy", "endfused"):
            return _Kernel(lambda f, ux, uy, rho, mask, W, H, u, stream=None:
                           macro(f, ux, uy, rho, mask, W, H, u, stream), name)
        raise AttributeError(f"{k} module has no kernel {name!r}")
