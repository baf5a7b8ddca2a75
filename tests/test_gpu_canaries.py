"""Out-of-bounds write detection without a sanitizer: every device array an entry
point receives sits between two 16 KB guard regions filled with a fixed bit
pattern; after the call the guards must be intact and the read-only inputs
(the source state of a ping-pong step, the mask) unchanged.  Covers the
drop-ins (tile kernel alone and the split launch), the general solver at every
depth, the in-place stepping, the diagnostics (the no-allocation one too), the
batch and the learned closure, on aligned and unaligned widths."""
import numpy as np
import pytest
import torch

import lbm_b200 as L
from lbm_b200 import _lib
from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu

GUARD_BYTES = 16384
PATTERN = {torch.float32: 0x7FC0DEAD, torch.float16: 0x7E5A, torch.bfloat16: 0x7FDA, torch.uint8: 0xA5,
           torch.float64: 0x7FF8DEADBEEFCAFE}
INT = {torch.float32: torch.int32, torch.float16: torch.int16, torch.bfloat16: torch.int16, torch.uint8: torch.uint8,
       torch.float64: torch.int64}


class Guarded:
    """A device array of `shape` between two guard regions; `t` is the array."""

    def __init__(self, shape, dtype, init=None):
        self.dtype = dtype
        esz = torch.tensor([], dtype=dtype).element_size()
        self.g = GUARD_BYTES // esz
        self.n = int(np.prod(shape))
        pat = PATTERN[dtype]
        itype = INT[dtype]
        if itype == torch.int16 and pat >= 1 << 15:
            pat -= 1 << 16
        self.raw = torch.full((2 * self.g + self.n,), pat, dtype=itype, device="cuda")
        self.pat = pat
        self.t = self.raw[self.g:self.g + self.n].view(dtype).view(*shape)
        if init is not None:
            self.t.copy_(torch.as_tensor(init).to(device="cuda", dtype=dtype).view(*shape))
        else:
            self.t.zero_()
        assert self.t.data_ptr() % 16 == 0

    def check(self, what):
        torch.cuda.synchronize()
        lo = self.raw[:self.g]
        hi = self.raw[self.g + self.n:]
        assert bool((lo == self.pat).all()) and bool((hi == self.pat).all()), f"{what}: guard overwritten"


def _case(W, H, seed=1):
    m = I.random_discs_mask(W, H, 3, 3.0, 7.0, seed, value=I.OBSTACLE)
    f0 = I.perturbed_state(W, H, seed + 3, amp=0.02)
    return m, f0


def _arrays(W, H, m, f0, dtype=torch.float32):
    mask = Guarded((H, W), torch.uint8, m)
    fa = Guarded((9, H, W), dtype)
    fb = Guarded((9, H, W), dtype)
    mac = [Guarded((H, W), torch.float32) for _ in range(3)]
    return mask, fa, fb, mac


@pytest.mark.parametrize("W,H", [(130, 66), (256, 96), (2048, 2048)])
def test_dropins_stay_in_bounds(W, H):
    m, f0 = _case(W, H)
    mask, fa, fb, mac = _arrays(W, H, m, f0)
    fa.t.copy_(torch.from_numpy(f0))
    mk = mask.t.clone()
    u = [g.t for g in mac]
    L.core4_step(mask.t, fa.t, fb.t, *u, W, H, 1.8, 0.1)
    L.smemaa_step(mask.t, fa.t, fb.t, *u, W, H, 1.7, 0.1, T=4)
    L.blocked_step(mask.t, fa.t, fb.t, W, H, 1.7, 0.1, T=6)
    L.smemaa_step(mask.t, fa.t, fb.t, *u, W, H, 1.7, 0.1, T=2)
    L.macro(fb.t, *u, mask.t, W, H, 0.1)
    img = Guarded((H, W, 4), torch.uint8)
    L.visualize(u[0], u[1], u[2], img.t, mask.t, W, H, 50.0)
    L.core4_run(mask.t, fa.t, fb.t, *u, W, H, 1.8, 0.1, 8, 4)
    for g, name in ((mask, "mask"), (fb, "f_out"), (img, "image")) + tuple((g, "macro") for g in mac):
        g.check(name)
    fa.check("f_a")
    torch.cuda.synchronize()
    assert torch.equal(mask.t, mk), "the mask was written"


@pytest.mark.parametrize("storage,dtype", [(SV.STORE_F32, torch.float32), (SV.STORE_F16DEV, torch.float16)])
@pytest.mark.parametrize("W,H", [(130, 66), (256, 96), (640, 200), (600, 200)])  # 600: padded mask rows
def test_general_solver_stays_in_bounds(W, H, storage, dtype):
    m, f0 = _case(W, H, 5)
    mask, fa, fb, mac = _arrays(W, H, m, f0, dtype)
    f32 = torch.from_numpy(f0).cuda()
    SV.convert_state(f32, SV.STORE_F32, fa.t, storage)
    S = SV.Solver(W, H, storage=storage, cs_smag=0.1, u_in=0.05, s_nu=1.9)
    u = [g.t for g in mac]
    for T in (1, 2, 3, 4, 5, 6, 8):
        src = fa.t.clone()
        S.run(fa.t, fb.t, mask.t, T, T, *u)  # one launch: f_a is the source only
        torch.cuda.synchronize()
        assert torch.equal(fa.t, src), f"T={T}: the source state was written"
        fb.check(f"T={T} f_out")
    S.run_inplace(fb.t, mask.t, 6, *u)
    fb.check("in place")
    out = Guarded((3,), torch.float64)
    S.diag(fb.t, mask.t, out=out.t)
    out.check("diag")
    frc = Guarded((2,), torch.float64)
    S.forces(fb.t, mask.t, out=frc.t)
    frc.check("forces")
    out2 = Guarded((3,), torch.float64)
    _lib.call("lbm_diag_fp64_noalloc", W, H, int(storage), L._ptr(fb.t), L._ptr(mask.t), L._ptr(out2.t),
              L._stream(None))
    out2.check("noalloc diag")
    for g in [mask, fa] + mac:
        g.check("input / macro")
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.t.cpu().numpy(), out2.t.cpu().numpy(), rtol=1e-12)


def test_batch_and_learned_closure_stay_in_bounds():
    from lbm_b200.batch import Batch
    from lbm_b200.closure import Mlp

    doms, keep = [], []
    for i, (W, H) in enumerate([(128, 64), (200, 96), (320, 72)]):
        m, f0 = _case(W, H, 10 + i)
        mask, fa, fb, _ = _arrays(W, H, m, f0, torch.float16)
        SV.convert_state(torch.from_numpy(f0).cuda(), SV.STORE_F32, fa.t, SV.STORE_F16DEV)
        fb.t.copy_(fa.t)
        doms.append(dict(W=W, H=H, f_a=fa.t, f_b=fb.t, mask=mask.t, u_in=0.05))
        keep.append((mask, fa, fb))
    B = Batch(doms, storage=SV.STORE_F16DEV, cs_smag=0.1, s_nu=1.9)
    for T in (1, 2, 4):
        B.run(2 * T, T)
    for mask, fa, fb in keep:
        mask.check("batch mask")
        fa.check("batch f_a")
        fb.check("batch f_b")
    W, H = 256, 96
    m, f0 = _case(W, H, 7)
    mask, fa, fb, mac = _arrays(W, H, m, f0)
    fa.t.copy_(torch.from_numpy(f0))
    net = Mlp(seed=0, in_scale=np.full(5, 1e3, np.float32), out_scale=1e-4)
    S = SV.Solver(W, H, closure=SV.CLOSURE_MLP, mlp=net.packed().data_ptr(), ref_clamps=0, u_in=0.05, s_nu=1.9)
    u = [g.t for g in mac]
    for T in (1, 2, 3, 4):
        S.run(fa.t, fb.t, mask.t, T, T, *u)
        fb.check(f"mlp T={T}")
    for g in [mask, fa] + mac:
        g.check("mlp input / macro")
