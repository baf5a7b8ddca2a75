"""lbm_diag_fp64_noalloc: the FP64 mass / momentum reduction with its scratch in a
fixed array inside the library (no cudaMalloc), against lbm_diag_fp64 (handle
scratch from lbm_create) on the same states, two calls in a row.  Collected last
so that it also runs after every other test in the same process."""
import ctypes as C

import numpy as np
import pytest
import torch

import lbm_b200 as L
from helpers import REL_TOL, dev
from lbm_b200 import init as I
from lbm_b200 import solver as SV

ERR_ARG, ERR_TOO_LARGE = 1001, 1005
MAX_CELLS = 134217728
TDT = {SV.STORE_F32: torch.float32, SV.STORE_F16DEV: torch.float16, SV.STORE_BF16DEV: torch.bfloat16}


def _noalloc(W, H, storage, f, mask, out, stream=None):
    return L.lib().lbm_diag_fp64_noalloc(W, H, storage, L._ptr(f), L._ptr(mask), L._ptr(out), L._stream(stream))


def _state(W, H, storage, seed):
    m = I.random_discs_mask(W, H, 3, 4.0, 9.0, seed)
    f32 = dev(I.perturbed_state(W, H, seed, amp=0.02))
    f = torch.empty((9, H, W), dtype=TDT[storage], device="cuda")
    SV.convert_state(f32, SV.STORE_F32, f, storage)
    return f, dev(m)


def _close(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return np.abs(a - b).max() <= REL_TOL * np.abs(b).max()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV, SV.STORE_BF16DEV])
def test_noalloc_matches_diag_two_calls(storage):
    # the second domain is smaller, so partials left by the first call lie
    # beyond what the second call reads; a stale block counter would also show
    cases = [(1030, 517, 11), (333, 97, 12)]
    results = []
    for W, H, seed in cases:
        f, m = _state(W, H, storage, seed)
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(W, H, storage, f, m, out) == 0
        S = SV.Solver(W, H, storage=storage)
        ref = S.diag(f, m)
        torch.cuda.synchronize()
        S.close()
        results.append((out.clone(), ref.clone()))
    for out, ref in results:
        assert torch.isfinite(out).all()
        assert _close(out, ref), (out, ref)
    # the two states differ, and so do their sums
    assert not torch.equal(results[0][0], results[1][0])


@pytest.mark.gpu
def test_noalloc_at_the_size_limit():
    """Exactly LBM_NOALLOC_MAX_CELLS cells (16384 x 8192, FP16 storage): every
    partial slot of the fixed array is used and the last block's counter
    comparison is at its maximum.  Two calls in a row give the same sums (the
    block counter is back at zero after the first), equal to lbm_diag_fp64."""
    W, H = 16384, MAX_CELLS // 16384
    g = torch.Generator(device="cuda").manual_seed(5)
    f = (0.01 * torch.randn((9, H, W), generator=g, device="cuda")).to(torch.float16)
    m = (torch.rand((H, W), generator=g, device="cuda") < 0.1).to(torch.uint8)
    outs = []
    for _ in range(2):
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(W, H, SV.STORE_F16DEV, f, m, out) == 0
        outs.append(out)
    S = SV.Solver(W, H, storage=SV.STORE_F16DEV)
    ref = S.diag(f, m)
    torch.cuda.synchronize()
    S.close()
    assert torch.equal(outs[0], outs[1])
    assert torch.isfinite(outs[0]).all()
    assert _close(outs[0], ref), (outs[0], ref)
    del f, m
    torch.cuda.empty_cache()


@pytest.mark.gpu
def test_noalloc_rejects_domain_above_limit():
    # real buffers of the rejected size, so nothing could be read out of bounds
    W, H = 16384, MAX_CELLS // 16384 + 1
    f = torch.empty((9, H, W), dtype=torch.float16, device="cuda")
    m = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    assert _noalloc(W, H, SV.STORE_F16DEV, f, m, out) == ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert torch.equal(out, torch.zeros_like(out))
    del f, m
    torch.cuda.empty_cache()


def test_noalloc_validation_before_any_device_call():
    if torch.cuda.is_available():
        pytest.skip("passes placeholder pointers; runs where no GPU is present")
    lib = L.lib()
    p = C.c_void_p(256)
    assert lib.lbm_diag_fp64_noalloc(16384, MAX_CELLS // 16384 + 1, SV.STORE_F32, p, p, p, None) == ERR_TOO_LARGE
    assert lib.lbm_diag_fp64_noalloc(0, 8, SV.STORE_F32, p, p, p, None) == ERR_ARG
    assert lib.lbm_diag_fp64_noalloc(8, 8, 7, p, p, p, None) == ERR_ARG
    assert lib.lbm_diag_fp64_noalloc(8, 8, SV.STORE_F32, None, p, p, None) == ERR_ARG
    assert b"LBM_NOALLOC_MAX_CELLS" in lib.lbm_error_string(ERR_TOO_LARGE)
