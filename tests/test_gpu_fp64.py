"""GPU tests of FP64 storage (LBM_STORE_F64: double planes, double arithmetic,
one step per launch), the high-precision judge of the other formats.

* against the FP64 CPU oracle on every boundary configuration of the general
  solver and on the full 4096 x 1024 cylinder channel: relative L2 <= 1e-12 on
  the populations (both sides compute in double; they differ only by the
  rounding of contracted multiply-adds), u, v, rho (written as float) <= 1e-6;
* the format-generic helpers in FP64 (equilibrium, conversion, reductions);
* a reduced configuration of the 8192 x 2048 storage study (2048 x 512, D = 64
  cylinder, the same inlet velocity and viscosity, 1000 steps): FP32, FP16 and
  BF16 storage against this judge, each with its error bound."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import dev, host, rel_l2
from lbm_b200 import LbmError
from lbm_b200 import init as I
from lbm_b200 import solver as SV
from test_gpu_general import BCS, CASES, case_inputs

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
MACRO_TOL = 1e-6  # u, v, rho leave the kernel as float


def f32(x):
    """The float32 value the C ABI receives for a parameter (lbm_params holds floats)."""
    return float(np.float32(x))


def make64(W, H, collision="mrt", closure="smag", s_nu=1.8, s_e=1.1, s_eps=1.1, s_q=1.1, cs=0.2,
           bc_left="zouhe_ramp", bc_right="outflow", bc_y="wall", u_in=0.1, u_lid=0.0, ref_clamps=True):
    S = SV.Solver(W, H, storage=SV.STORE_F64, collision=SV.COLL_MRT if collision == "mrt" else SV.COLL_BGK,
                  closure=SV.CLOSURE_SMAG if closure == "smag" else SV.CLOSURE_NONE, s_nu=s_nu, s_e=s_e, s_eps=s_eps,
                  s_q=s_q, cs_smag=cs, bc_left=BCS[bc_left], bc_right=BCS[bc_right], bc_y=BCS[bc_y], u_in=u_in,
                  u_lid=u_lid, ref_clamps=int(ref_clamps))
    G = O.General(W, H, collision=collision, closure=closure, s_nu=f32(s_nu), s_e=f32(s_e), s_eps=f32(s_eps),
                  s_q=f32(s_q), cs=f32(cs), bc_left=bc_left, bc_right=bc_right, bc_y=bc_y, u_in=f32(u_in),
                  u_lid=f32(u_lid), ref_clamps=ref_clamps)
    return S, G


@pytest.mark.parametrize("W,H", [(130, 66), (256, 96)])
@pytest.mark.parametrize("name", list(CASES))
def test_f64_vs_fp64_oracle(name, W, H):
    kw, kind = CASES[name]
    S, G = make64(W, H, **kw)
    m, f0 = case_inputs(kind, W, H)
    f0 = f0.astype(np.float64)
    n = 24
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    which = S.run(a, b, dev(m), n, 2, *mac)  # T is ignored in FP64: one step per launch
    assert which == n % 2
    out = host(b if which else a)
    ref, rmac = G.run(m, f0, n)
    assert rel_l2(out, ref) < F64_TOL, rel_l2(out, ref)
    upd = m == 0
    for g_, r_ in zip(mac, rmac):
        assert rel_l2(host(g_)[upd], r_[upd]) < MACRO_TOL


def test_f64_channel_4096x1024_vs_fp64_oracle():
    """The bench workload's physics (MRT + Smagorinsky Cs = 0.1, clamps, ramped
    Zou-He inlet, outflow, D = 128 cylinder) at its full size, from a perturbed
    state, 24 steps."""
    W, H, n = 4096, 1024, 24
    kw = dict(cs=0.1, u_in=0.05, s_nu=1.0 / 0.50192)
    S, G = make64(W, H, **kw)
    m = I.cylinder_mask(W, H, 1024, 512, 128, value=I.OBSTACLE)
    f0 = I.perturbed_state(W, H, 21, amp=0.02).astype(np.float64)
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    which = S.run(a, b, dev(m), n, 1, *mac)
    out = host(b if which else a)
    ref, rmac = G.run(m, f0, n)
    assert rel_l2(out, ref) < F64_TOL, rel_l2(out, ref)
    upd = m == 0
    for g_, r_ in zip(mac, rmac):
        assert rel_l2(host(g_)[upd], r_[upd]) < MACRO_TOL
    S.close()


def test_f64_helpers():
    W, H = 200, 70
    S = SV.Solver(W, H, storage=SV.STORE_F64, ref_clamps=0, closure=SV.CLOSURE_NONE, bc_left=SV.BC_WALL,
                  bc_right=SV.BC_WALL)
    assert int(SV.lib().lbm_state_bytes(S.handle)) == 9 * W * H * 8
    # equilibrium in double: rho = 1 + 0.01, u = (0.03, -0.02) everywhere
    rho = torch.full((H, W), 1.01, device="cuda")
    ux = torch.full((H, W), 0.03, device="cuda")
    uy = torch.full((H, W), -0.02, device="cuda")
    f = S.new_state()
    S.init_equilibrium(f, rho, ux, uy)
    r, u, v = np.float64(np.float32(1.01)), np.float64(np.float32(0.03)), np.float64(np.float32(-0.02))
    want = np.array([I.WEIGHTS[q] * r * (1 + 3 * (I.CX[q] * u + I.CY[q] * v) + 4.5 * (I.CX[q] * u + I.CY[q] * v) ** 2
                                   - 1.5 * (u * u + v * v)) for q in range(9)])
    np.testing.assert_allclose(host(f)[:, 3, 5], want, rtol=1e-14)
    # conversion: FP32 -> FP64 is exact, and back again
    x32 = dev(I.perturbed_state(W, H, 4, amp=0.02))
    x64 = S.new_state()
    SV.convert_state(x32, SV.STORE_F32, x64, SV.STORE_F64)
    assert torch.equal(x64, x32.double())
    back = torch.empty_like(x32)
    SV.convert_state(x64, SV.STORE_F64, back, SV.STORE_F32)
    assert torch.equal(back, x32)
    # FP64 reductions of a double state equal host sums
    m = dev(I.random_discs_mask(W, H, 3, 3.0, 6.0, 5))
    d = host(S.diag(x64, m))
    f64 = host(x64)
    fl = host(m) == 0
    want = [f64[:, fl].sum(), (f64 * I.CX[:, None, None])[:, fl].sum(), (f64 * I.CY[:, None, None])[:, fl].sum()]
    np.testing.assert_allclose(d, want, rtol=1e-13, atol=1e-12)
    # one state buffer is not built for FP64
    with pytest.raises(LbmError):
        S.run_inplace(x64, m, 2)
    S.close()


# Reduced configuration of the storage-format study: the 8192 x 2048 cylinder
# channel at a quarter of the size in each direction (D = 64, Re = 5000).
C3R = dict(cs_smag=0.1, u_in=0.05, s_nu=1.0 / (3.0 * 6.4e-4 + 0.5))
# Measured on a B200: FP32 1.1e-4, FP16 3.4e-3, BF16 3.6e-2 (the flow from rest
# amplifies rounding: FP32 is 1e-6 from FP64 after 8 steps, 1e-4 after 1000).
C3R_BOUNDS = {"f32": 5e-4, "f16": 1e-2, "bf16": 8e-2}


def test_reduced_storage_study_vs_fp64_judge():
    W, H, n = 2048, 512, 1000
    mask = dev(I.cylinder_mask(W, H, 512, 256, 64, value=I.OBSTACLE))
    f0 = dev(I.channel_state(W, H, u0=0.0, noise=1e-4, seed=0))
    fl = host(mask) == 0
    vel = {}
    for name, st in (("f64", SV.STORE_F64), ("f32", SV.STORE_F32), ("f16", SV.STORE_F16DEV),
                     ("bf16", SV.STORE_BF16DEV)):
        S = SV.Solver(W, H, storage=st, **C3R)
        a = S.new_state()
        SV.convert_state(f0, SV.STORE_F32, a, st)
        b = a.clone()
        mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
        S.run(a, b, mask, n, 2, *mac)
        vel[name] = np.stack([host(mac[0]), host(mac[1])])[:, fl].astype(np.float64)
        S.close()
    errs = {k: rel_l2(vel[k], vel["f64"]) for k in ("f32", "f16", "bf16")}
    print("2048x512 cylinder, 1000 steps, velocity rel L2 vs FP64:", errs)
    for k, bound in C3R_BOUNDS.items():
        assert errs[k] < bound, (k, errs[k])
    assert errs["f32"] < errs["f16"] < errs["bf16"]
