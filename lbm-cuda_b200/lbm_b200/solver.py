"""General solver (lbm_params / lbm_create / lbm_run) with torch device arrays."""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import call, lib

STORE_F32, STORE_F16DEV, STORE_BF16DEV, STORE_F64 = 0, 1, 2, 3
COLL_BGK, COLL_MRT = 0, 1
CLOSURE_NONE, CLOSURE_SMAG, CLOSURE_MLP, CLOSURE_MLP_SILU = 0, 1, 2, 3
BC_WALL, BC_PERIODIC, BC_ZOUHE, BC_ZOUHE_RAMP, BC_OUTFLOW = 0, 1, 2, 3, 4


class Params(C.Structure):
    """Mirror of ``lbm_params`` (include/lbm_b200.h)."""

    _fields_ = [
        ("W", C.c_int), ("H", C.c_int), ("storage", C.c_int), ("collision", C.c_int), ("closure", C.c_int),
        ("s_nu", C.c_float), ("s_e", C.c_float), ("s_eps", C.c_float), ("s_q", C.c_float),
        ("cs_smag", C.c_float), ("bc_left", C.c_int), ("bc_right", C.c_int), ("bc_y", C.c_int),
        ("u_in", C.c_float), ("u_lid", C.c_float), ("ref_clamps", C.c_int), ("mlp", C.c_void_p),
    ]


def default_params(W: int, H: int, **overrides) -> Params:
    p = Params()
    lib().lbm_params_default(C.byref(p), int(W), int(H))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"lbm_params has no field {k!r}")
        setattr(p, k, v)
    return p


def _torch_dtype(storage: int):
    import torch

    return {STORE_F32: torch.float32, STORE_F16DEV: torch.float16, STORE_BF16DEV: torch.bfloat16,
            STORE_F64: torch.float64}[storage]


class Solver:
    """Owns an lbm_handle.  States are torch tensors shaped (9, H, W) in the
    handle's storage format (float32, float16/bfloat16 holding f_q - w_q, or
    float64: the FP64 judge, one step per launch whatever T)."""

    def __init__(self, W: int, H: int, params: Params | None = None, **overrides):
        self.params = params if params is not None else default_params(W, H, **overrides)
        self.W, self.H = int(self.params.W), int(self.params.H)
        h = C.c_void_p(0)
        call("lbm_create", C.byref(self.params), C.byref(h))
        self._h = h

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("solver is closed")
        return self._h

    def close(self) -> None:
        if self._h:
            call("lbm_destroy", self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dtype(self):
        return _torch_dtype(self.params.storage)

    def new_state(self):
        import torch

        return torch.empty((9, self.H, self.W), dtype=self.dtype, device="cuda")

    def init_equilibrium(self, f, rho=None, ux=None, uy=None, stream=None):
        from . import _ptr, _stream

        call("lbm_init_equilibrium", self.handle, _ptr(f), _ptr(rho), _ptr(ux), _ptr(uy), _stream(stream))

    def run(self, f_a, f_b, mask, n_steps: int, T: int = 2, ux=None, uy=None, rho=None, stream=None) -> int:
        """n_steps steps fused T per launch; returns 1 when the result is in f_b.  The
        default T = 2 is the fastest depth measured on a B200 for domains larger
        than the L2 cache (the register wavefront; T = 3 is close).  Domains periodic
        in x advance one step per launch whatever T (the faster kernel there; the
        slab layer runs them on the register wavefront with halo columns)."""
        from . import _ptr, _stream

        out = C.c_int(0)
        call("lbm_run", self.handle, _ptr(f_a), _ptr(f_b), _ptr(mask), int(n_steps), int(T), _ptr(ux), _ptr(uy),
             _ptr(rho), _stream(stream), C.byref(out))
        return out.value

    def run_columns(self, f_a, f_b, mask, T: int, x0: int, x1: int, stream=None) -> None:
        """lbm_run_columns: one launch of T steps f_a -> f_b writing only columns [x0, x1) of f_b."""
        from . import _ptr, _stream

        call("lbm_run_columns", self.handle, _ptr(f_a), _ptr(f_b), _ptr(mask), int(T), int(x0), int(x1),
             _stream(stream))

    def reset_graphs(self) -> None:
        """lbm_run_graph_reset: drop the cached launch-pair graphs (call before
        freeing state buffers whose addresses new buffers may reuse)."""
        call("lbm_run_graph_reset", self.handle)

    def run_checked(self, f_a, f_b, mask, n_steps: int, T: int = 2, check_every: int = 1000, ux=None, uy=None,
                    rho=None, stream=None) -> int:
        """lbm_run in chunks of check_every steps; after each chunk the FP64 mass
        and momentum (lbm_diag_fp64) of the state must be finite, else
        FloatingPointError names the steps in which it stopped being finite (the
        device-side failure detection: one small reduction and one host read per
        chunk).  Returns 1 when the final state is in f_b, like run."""
        import math

        cur, oth = f_a, f_b
        done = 0
        while done < n_steps:
            k = min(int(check_every), n_steps - done)
            last = done + k == n_steps
            which = self.run(cur, oth, mask, k, T, *((ux, uy, rho) if last else (None, None, None)), stream=stream)
            if which:
                cur, oth = oth, cur
            d = self.diag(cur, mask, stream=stream).cpu().tolist()
            if not all(math.isfinite(x) for x in d):
                raise FloatingPointError(f"the state is not finite after steps {done + 1}..{done + k} "
                                         f"(mass, momentum = {d})")
            done += k
        return 1 if cur is f_b else 0

    def run_inplace(self, f, mask, n_steps: int, ux=None, uy=None, rho=None, stream=None) -> None:
        """lbm_run_inplace: n_steps (even) steps in the single state buffer f."""
        from . import _ptr, _stream

        call("lbm_run_inplace", self.handle, _ptr(f), _ptr(mask), int(n_steps), _ptr(ux), _ptr(uy), _ptr(rho),
             _stream(stream))

    def diag(self, f, mask, out=None, stream=None):
        """Device tensor [mass, momentum_x, momentum_y] (float64), fixed-order reduction."""
        import torch

        from . import _ptr, _stream

        out = torch.empty(3, dtype=torch.float64, device="cuda") if out is None else out
        call("lbm_diag_fp64", self.handle, _ptr(f), _ptr(mask), _ptr(out), _stream(stream))
        return out

    def forces(self, f, mask, out=None, stream=None):
        """Device tensor [drag, lift] (float64), momentum exchange on LBM_MASK_OBSTACLE cells."""
        import torch

        from . import _ptr, _stream

        out = torch.empty(2, dtype=torch.float64, device="cuda") if out is None else out
        call("lbm_forces_fp64", self.handle, _ptr(f), _ptr(mask), _ptr(out), _stream(stream))
        return out


def convert_state(src, src_storage: int, dst, dst_storage: int, stream=None) -> None:
    from . import _ptr, _stream

    _, H, W = src.shape
    call("lbm_convert_state", int(W), int(H), _ptr(src), int(src_storage), _ptr(dst), int(dst_storage),
         _stream(stream))


def halo_pack(f, storage: int, xl: int, xr: int, ncols: int, buf, stream=None) -> None:
    """lbm_halo_pack: columns [xl, xl + ncols) and [xr, xr + ncols) of every plane
    of f (9, H, width) into buf (2, 9, H, ncols); a negative start skips its side."""
    from . import _ptr, _stream

    _, H, width = f.shape
    call("lbm_halo_pack", _ptr(f), int(width), int(H), int(storage), int(xl), int(xr), int(ncols), _ptr(buf),
         _stream(stream))


def halo_unpack(f, storage: int, xl: int, xr: int, ncols: int, buf, stream=None) -> None:
    """lbm_halo_unpack: the reverse of halo_pack."""
    from . import _ptr, _stream

    _, H, width = f.shape
    call("lbm_halo_unpack", _ptr(f), int(width), int(H), int(storage), int(xl), int(xr), int(ncols), _ptr(buf),
         _stream(stream))


def device_error_flags(clear: bool = True) -> int:
    v = C.c_int(0)
    call("lbm_device_error_flags", C.byref(v), int(bool(clear)))
    return v.value


__all__ = ["Params", "Solver", "default_params", "convert_state", "device_error_flags", "_lib"]
