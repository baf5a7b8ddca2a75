"""Generate the golden fixtures in tests/golden/ from the reference's own kernels.

Runs on a machine with a B200: it loads oracle/_ref/libref_*.so (the reference's
.cu sources compiled by oracle/Makefile with -use_fast_math, as its drivers
compile them), runs them on seeded synthetic inputs with the drivers' launch
shapes and ping-pong buffer order, and writes one compressed .npz per case with
the inputs and the outputs after several launch counts.  The CPU oracle is
checked against these files by tests/test_oracle_golden.py.

    python tests/golden/make_golden.py [outdir]
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "lbm-cuda_b200"))
from lbm_b200 import init as lbinit  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def _lib(name):
    lib = C.CDLL(os.path.join(REF, name))
    return lib


def _ptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def policy_mask(W, H, seed):
    """Random discs in a channel (driver conventions).  The policy/endfused kernels
    read shared-memory slots they never initialise next to the outlet corners
    (W-1, 0) and (W-1, H-1); tests compare outside those corners' light cones."""
    return lbinit.random_discs_mask(W, H, 3, 3.0, 7.0, seed, value=1)


def core4_case(W, H, seed, snaps, tau_inv=1.8, u_in=0.1):
    lib = _lib("libref_core4.so")
    lib.ref_core4_step.argtypes = [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_void_p]
    mask = lbinit.random_discs_mask(W, H, 3, 3.0, 7.0, seed, value=1)
    f0 = lbinit.perturbed_state(W, H, seed + 10)
    m, a = _dev(mask), _dev(f0)
    b = a.clone()  # the driver's f_out = f_now.copy() (lbm_mine2.py:36)
    mac = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in range(3)]
    out = dict(mask=mask, f0=f0, W=W, H=H, tau_inv=tau_inv, u_in=u_in, snaps=np.array(snaps))
    for step in range(1, max(snaps) + 1):
        rc = lib.ref_core4_step(_ptr(m), _ptr(a), _ptr(b), *[_ptr(t) for t in mac], W, H, tau_inv, u_in, tau_inv,
                                _stream())
        assert rc == 0, rc
        a, b = b, a
        if step in snaps:
            torch.cuda.synchronize()
            out[f"f_{step}"] = a.cpu().numpy()
            for k, t in zip(("ux", "uy", "rho"), mac):
                out[f"{k}_{step}"] = t.cpu().numpy()
    return out


def smemaa_case(W, H, seed, launches, tau_inv=1.7, u_in=0.1):
    lib = _lib("libref_smemaa.so")
    lib.ref_smemaa_step.argtypes = [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p]
    T = lib.ref_T()
    mask = lbinit.random_discs_mask(W, H, 3, 3.0, 7.0, seed, value=1)
    f0 = lbinit.perturbed_state(W, H, seed + 10)
    m, a = _dev(mask), _dev(f0)
    b = a.clone()
    mac = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in range(3)]
    out = dict(mask=mask, f0=f0, W=W, H=H, T=T, tau_inv=tau_inv, u_in=u_in, snaps=np.array(launches))
    for n in range(1, max(launches) + 1):
        rc = lib.ref_smemaa_step(_ptr(m), _ptr(a), _ptr(b), *[_ptr(t) for t in mac], W, H, tau_inv, u_in, _stream())
        assert rc == 0, rc
        a, b = b, a
        if n in launches:
            torch.cuda.synchronize()
            out[f"f_{n}"] = a.cpu().numpy()
            for k, t in zip(("ux", "uy", "rho"), mac):
                out[f"{k}_{n}"] = t.cpu().numpy()
    return out


def blocked_case(libname, W, H, seed, launches, tau_inv=1.0, u_in=0.1):
    lib = _lib(libname)
    lib.ref_blocked_step.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p]
    lib.ref_macro.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_float, C.c_void_p]
    T = lib.ref_T()
    mask = policy_mask(W, H, seed)
    f0 = lbinit.perturbed_state(W, H, seed + 10)
    m, a = _dev(mask), _dev(f0)
    b = a.clone()  # deterministic stale contents for entries B-final never writes
    mac = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in range(3)]
    out = dict(mask=mask, f0=f0, W=W, H=H, T=T, tau_inv=tau_inv, u_in=u_in, snaps=np.array(launches))
    for n in range(1, max(launches) + 1):
        rc = lib.ref_blocked_step(_ptr(m), _ptr(a), _ptr(b), W, H, tau_inv, u_in, _stream())
        assert rc == 0, rc
        a, b = b, a
        if n in launches:
            rc = lib.ref_macro(_ptr(a), *[_ptr(t) for t in mac], _ptr(m), W, H, u_in, _stream())
            assert rc == 0, rc
            torch.cuda.synchronize()
            out[f"f_{n}"] = a.cpu().numpy()
            for k, t in zip(("ux", "uy", "rho"), mac):
                out[f"{k}_{n}"] = t.cpu().numpy()
    return out


def visualize_case(W, H, seed, vort_scale=50.0):
    lib = _lib("libref_core4.so")
    lib.ref_visualize.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_float, C.c_void_p]
    rng = np.random.default_rng(seed)
    mask = lbinit.random_discs_mask(W, H, 2, 3.0, 6.0, seed, value=1)
    ux = (0.02 * rng.standard_normal((H, W))).astype(np.float32)
    uy = (0.02 * rng.standard_normal((H, W))).astype(np.float32)
    rho = np.ones((H, W), np.float32)
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    keep = [_dev(ux), _dev(uy), _dev(rho), img, _dev(mask)]  # device arrays stay alive until the kernel ran
    rc = lib.ref_visualize(*[_ptr(t) for t in keep], W, H, vort_scale, _stream())
    assert rc == 0, rc
    torch.cuda.synchronize()
    return dict(mask=mask, ux=ux, uy=uy, W=W, H=H, vort_scale=vort_scale, img=img.cpu().numpy())


CASES = {
    "core4_64x48": lambda: core4_case(64, 48, 1, [1, 2, 5, 12]),
    "core4_130x66": lambda: core4_case(130, 66, 2, [1, 3, 12]),
    "smemaa_64x48": lambda: smemaa_case(64, 48, 3, [1, 2, 3]),
    "smemaa_130x66": lambda: smemaa_case(130, 66, 4, [1, 3]),
    "policy_64x48": lambda: blocked_case("libref_policy.so", 64, 48, 5, [1, 2]),
    "policy_130x66": lambda: blocked_case("libref_policy.so", 130, 66, 6, [1, 2]),
    "endfused_130x66": lambda: blocked_case("libref_endfused.so", 130, 66, 7, [1, 2]),
    "visualize_96x40": lambda: visualize_case(96, 40, 8),
}


def main(outdir: str) -> None:
    os.makedirs(outdir, exist_ok=True)
    for name, fn in CASES.items():
        data = fn()
        path = os.path.join(outdir, name + ".npz")
        np.savez_compressed(path, **data)
        print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
