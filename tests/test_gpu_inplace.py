"""In-place time stepping (lbm_run_inplace: one state buffer, AA access pattern)
against the ping-pong solver (lbm_run) and the general-solver oracle.

Checks, for every boundary configuration of the general-solver tests (Zou-He
inlet with and without the ramp, outflow ghost, obstacles, moving lid,
periodic sides) and each storage format: after an even number of steps the
single buffer holds the same state as lbm_run's result (relative L2 <= 1e-6 in
FP32, the two paths evaluate the same collision on the same inputs) and u, v,
rho of the last step agree (1e-5); FP32 against the oracle at the parity tolerance
1e-5; an obstacle touching the outlet's source column (x = W - 2, where the
ghost copy stops) keeps the equality; odd step counts and the learned closure
are refused."""
import numpy as np
import pytest
import torch

from helpers import REL_TOL, dev, host, rel_l2
from lbm_b200 import solver as SV
from lbm_b200._lib import LbmError
from test_gpu_general import CASES, case_inputs, make

pytestmark = pytest.mark.gpu


def _pair(S, m, f0, n, tdt=torch.float32, storage=SV.STORE_F32):
    H, W = m.shape
    f32 = dev(f0)
    a = torch.empty(f32.shape, dtype=tdt, device="cuda")
    SV.convert_state(f32, SV.STORE_F32, a, storage)
    b = a.clone()
    c = a.clone()
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    imac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    md = dev(m)
    which = S.run(a, b, md, n, 1, *mac)
    S.run_inplace(c, md, n, *imac)
    torch.cuda.synchronize()
    ref = (b if which else a).float().cpu().numpy()
    return ref, c.float().cpu().numpy(), [host(t) for t in mac], [host(t) for t in imac]


@pytest.mark.parametrize("W,H", [(130, 66), (256, 96)])
@pytest.mark.parametrize("name", list(CASES))
def test_inplace_equals_pingpong_and_oracle(name, W, H):
    kw, kind = CASES[name]
    S, G = make(W, H, **kw)
    m, f0 = case_inputs(kind, W, H)
    n = 10
    ref, got, mac, imac = _pair(S, m, f0, n)
    assert rel_l2(got, ref) < 1e-6
    upd = m == 0
    for g_, r_ in zip(imac, mac):  # u, v are small: rounding of the moments shows at 1e-6
        assert rel_l2(g_[upd], r_[upd]) < REL_TOL
    oref, omac = G.run(m, f0, n)
    assert rel_l2(got, oref) < REL_TOL
    for g_, r_ in zip(imac, omac):
        assert rel_l2(g_[upd], np.asarray(r_)[upd]) < REL_TOL


@pytest.mark.parametrize("storage,tdt", [(SV.STORE_F16DEV, torch.float16), (SV.STORE_BF16DEV, torch.bfloat16)])
@pytest.mark.parametrize("name", ["mrt_smag_clamps_ramp", "mrt_periodic_y_channel"])
def test_inplace_16bit_storage(name, storage, tdt):
    W, H = 256, 96
    kw, kind = CASES[name]
    S, _ = make(W, H, storage=storage, **kw)
    m, f0 = case_inputs(kind, W, H)
    ref, got, mac, imac = _pair(S, m, f0, 12, tdt, storage)
    assert rel_l2(got, ref) < 1e-6
    upd = m == 0
    for g_, r_ in zip(imac, mac):
        assert rel_l2(g_[upd], r_[upd]) < 1e-5


@pytest.mark.parametrize("name", list(CASES))
def test_inplace_vector_path(name):
    """640 columns (W % 4 == 0): warps whose 128 cells are interior fluid take the
    vector path (128-bit accesses, warp-shuffled column shifts), the others the
    per-cell code; the state must equal lbm_run's."""
    W, H = 640, 96
    kw, kind = CASES[name]
    S, _ = make(W, H, **kw)
    m, f0 = case_inputs(kind, W, H, seed=3)
    ref, got, mac, imac = _pair(S, m, f0, 20)
    assert rel_l2(got, ref) < 1e-6
    upd = m == 0
    for g_, r_ in zip(imac, mac):
        assert rel_l2(g_[upd], r_[upd]) < REL_TOL


@pytest.mark.parametrize("storage,tdt", [(SV.STORE_F16DEV, torch.float16), (SV.STORE_BF16DEV, torch.bfloat16)])
def test_inplace_vector_path_16bit(storage, tdt):
    W, H = 640, 96
    kw, kind = CASES["mrt_smag_clamps_ramp"]
    S, _ = make(W, H, storage=storage, **kw)
    m, f0 = case_inputs(kind, W, H, seed=3)
    ref, got, _, _ = _pair(S, m, f0, 20, tdt, storage)
    assert rel_l2(got, ref) < 1e-6


def test_inplace_obstacle_at_the_outlet_source_column():
    """Solid cells at x = W - 2 (the ghost column's source) on some rows: those
    rows' ghost cells are never copied and must keep their values."""
    W, H = 128, 64
    kw, _ = CASES["mrt_smag_flat_inlet"]
    S, G = make(W, H, **kw)
    m, f0 = case_inputs("discs", W, H, seed=4)
    m[20:30, W - 2] = 3
    m[40, W - 3:W - 1] = 1
    ref, got, _, _ = _pair(S, m, f0, 16)
    assert rel_l2(got, ref) < 1e-6
    oref, _ = G.run(m, f0, 16)
    assert rel_l2(got, oref) < REL_TOL


def test_inplace_long_run_matches():
    """2000 steps of the cylinder-channel physics at 512 x 128: the in-place
    state stays equal to the ping-pong state (same arithmetic on every step)."""
    W, H = 512, 128
    kw, kind = CASES["mrt_smag_clamps_ramp"]
    S, _ = make(W, H, **kw)
    m, f0 = case_inputs(kind, W, H, seed=2)
    ref, got, _, _ = _pair(S, m, f0, 2000)
    assert rel_l2(got, ref) < 1e-5


def test_inplace_refuses_odd_steps_and_the_learned_closure():
    W, H = 64, 32
    S, _ = make(W, H, **CASES["mrt_smag_clamps_ramp"][0])
    f = torch.zeros((9, H, W), device="cuda")
    m = torch.zeros((H, W), dtype=torch.uint8, device="cuda")
    with pytest.raises(LbmError):
        S.run_inplace(f, m, 3)
    from lbm_b200.closure import Mlp

    net = Mlp(seed=0)
    Sm = SV.Solver(W, H, closure=SV.CLOSURE_MLP, mlp=net.packed().data_ptr(), ref_clamps=0)
    with pytest.raises(LbmError):
        Sm.run_inplace(f, m, 2)
