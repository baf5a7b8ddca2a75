"""Batched independent domains (lbm_batch_*): many domains of uneven size
advance together in one persistent launch per T steps."""
from __future__ import annotations

import ctypes as C

from ._lib import call
from .solver import Params, default_params

SIZE_CLASSES = 3  # LBM_BATCH_SIZE_CLASSES: < 2^17 cells, < 2^19, larger


class Domain(C.Structure):
    """Mirror of ``lbm_domain`` (include/lbm_b200.h)."""

    _fields_ = [("W", C.c_int), ("H", C.c_int), ("pitch", C.c_int), ("mask_pitch", C.c_int), ("f_a", C.c_void_p),
                ("f_b", C.c_void_p), ("mask", C.c_void_p), ("u_in", C.c_float)]


class Batch:
    """Owns an lbm_batch.  ``domains`` is a list of dicts with keys W, H, f_a, f_b,
    mask (torch device tensors), u_in and optionally pitch / mask_pitch."""

    def __init__(self, domains, params: Params | None = None, **overrides):
        from . import _ptr

        self.params = params if params is not None else default_params(1, 1, **overrides)
        arr = (Domain * len(domains))()
        self._keep = []
        for i, d in enumerate(domains):
            arr[i].W, arr[i].H = int(d["W"]), int(d["H"])
            arr[i].pitch = int(d.get("pitch", 0))
            arr[i].mask_pitch = int(d.get("mask_pitch", 0))
            arr[i].f_a = _ptr(d["f_a"]).value
            arr[i].f_b = _ptr(d["f_b"]).value
            arr[i].mask = _ptr(d["mask"]).value
            arr[i].u_in = float(d.get("u_in", self.params.u_in))
            self._keep.append(d)
        h = C.c_void_p(0)
        call("lbm_batch_create", C.byref(self.params), arr, len(domains), C.byref(h))
        self._h = h

    def close(self):
        if self._h:
            call("lbm_batch_destroy", self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n_steps: int, T: int = 0, stream=None) -> int:
        """Persistent batched launches; returns 1 when the states end in f_b."""
        from . import _stream

        out = C.c_int(0)
        call("lbm_batch_run", self._h, int(n_steps), int(T), _stream(stream), C.byref(out))
        return out.value

    def run_separate(self, n_steps: int, T: int = 4, stream=None) -> int:
        """The same steps with one launch per domain (comparison point)."""
        from . import _stream

        out = C.c_int(0)
        call("lbm_batch_run_separate", self._h, int(n_steps), int(T), _stream(stream), C.byref(out))
        return out.value

    def autotune(self, stream=None):
        """Pick T and the rows per work item of every size class; returns (T, rows of
        the largest populated class) (``tiles()`` gives all).  Synchronous;
        advances the states."""
        from . import _stream

        t, c = C.c_int(0), C.c_int(0)
        call("lbm_batch_autotune", self._h, _stream(stream), C.byref(t), C.byref(c))
        return t.value, c.value

    def tiles(self):
        """(T, [rows per item of each size class]) that run(T=0) uses."""
        t = C.c_int(0)
        rows = (C.c_int * SIZE_CLASSES)()
        call("lbm_batch_get_tiles", self._h, C.byref(t), rows)
        return t.value, list(rows)

    def set_tiles(self, T: int, rows) -> None:
        """Sets the configuration run(T=0) uses: depth T and rows per class."""
        arr = (C.c_int * SIZE_CLASSES)(*[int(r) for r in rows])
        call("lbm_batch_set_tiles", self._h, int(T), arr)
