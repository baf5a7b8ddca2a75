"""GPU tests of the learned closure: the training kernels (forward, gradient,
Adam) against the FP64 oracle, and the solver with LBM_CLOSURE_MLP (BF16 tensor-
core inference inside the register wavefront kernel) against the oracle's FP64
network.  Tolerance of the closure runs: relative L2 1e-4 on the populations
(BF16 weights and activations change nu_t by about 1 %, which moves a relaxation
rate by about 1e-5)."""
import numpy as np
import pytest
import torch

import mlp_oracle as MO
import oracle as O
from helpers import dev, host, rel_l2
from lbm_b200 import closure as CL
from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu


def _params(seed):
    rng = np.random.default_rng(seed)
    return CL.init_params(seed) + (0.05 * rng.standard_normal(CL.NPARAM)).astype(np.float32)


@pytest.mark.parametrize("act", ["relu", "silu"])
def test_forward_and_gradient_match_oracle(act):
    p = _params(1)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((5000, 5)).astype(np.float32)
    t = rng.random(5000).astype(np.float32)
    net = CL.Mlp(params=p, act=act)
    y = host(net.forward(dev(x)))
    yo, _ = MO.forward(p, x, act)
    assert np.abs(y - yo).max() <= 1e-5 * max(1.0, np.abs(yo).max())
    loss, g, _ = net.loss_grad(dev(x), dev(t))
    lo, go = MO.loss_grad(p, x, t, act=act)
    assert abs(float(loss.item()) - lo) <= 1e-5 * lo
    assert rel_l2(host(g).astype(np.float64), go) < 1e-4
    # deterministic: the same inputs give the same bits
    _, g2, _ = net.loss_grad(dev(x), dev(t))
    assert torch.equal(g, g2)


def test_adam_step_matches_numpy():
    p = _params(3)
    net = CL.Mlp(params=p)
    g = np.random.default_rng(4).standard_normal(CL.NPARAM).astype(np.float32)
    net.adam(dev(g), lr=1e-2)
    m = 0.1 * g
    v = 0.001 * g * g
    want = p - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.allclose(host(net.params), want, rtol=1e-5, atol=1e-7)


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((20000, 5)).astype(np.float32) * np.array([1e-3, 1e-3, 1e-4, 1e-3, 1e-3], np.float32)
    nu = (0.01 * np.log1p(np.exp(300 * x[:, 3] + 100 * x[:, 0]))).astype(np.float32)
    net = CL.Mlp(seed=1)
    tr, va = net.fit(x, nu, epochs=60, batch=1024, lr=3e-3)  # about 1000 Adam steps
    assert va[-1] < 0.05 * va[0]
    pred = host(net.predict(x[:2000]))
    assert rel_l2(pred, nu[:2000]) < 0.1


CH = dict(collision="mrt", bc_left="zouhe_ramp", bc_right="outflow", bc_y="wall", ref_clamps=False, s_nu=1.8,
          u_in=0.05)


@pytest.mark.parametrize("act", ["relu", "silu"])
@pytest.mark.parametrize("T", [1, 2, 3, 4])
def test_mlp_closure_run_matches_oracle(T, act):
    W, H, n = 256, 80, 2 * T + 1
    p = _params(7)
    in_scale = np.array([300.0, 300.0, 1000.0, 300.0, 100.0], np.float32)
    out_scale = 0.002
    net = CL.Mlp(params=p, in_scale=in_scale, out_scale=out_scale, act=act)
    m = I.random_discs_mask(W, H, 3, 3.0, 6.0, 11)
    f0 = I.perturbed_state(W, H, 12, amp=0.02)
    SV.device_error_flags(clear=True)
    S = SV.Solver(W, H, collision=SV.COLL_MRT, closure=net.closure, bc_left=SV.BC_ZOUHE_RAMP,
                  bc_right=SV.BC_OUTFLOW, bc_y=SV.BC_WALL, ref_clamps=0, s_nu=1.8, u_in=0.05,
                  mlp=net.packed().data_ptr())
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    which = S.run(a, b, dev(m), n, T, *mac)
    out = host(b if which else a)
    assert SV.device_error_flags(clear=True) == 0
    O.set_mlp(p, in_scale, out_scale)
    ref, rmac = O.General(W, H, closure="mlp" if act == "relu" else "mlp_silu", **CH).run(m, f0.astype(np.float64),
                                                                                         n)
    assert rel_l2(out, ref) < 1e-4
    upd = m == 0
    for g_, r_ in zip(mac, rmac):
        assert rel_l2(host(g_)[upd], r_[upd]) < 1e-4


def test_mlp_closure_16bit_storage_runs():
    W, H, n = 256, 64, 10
    net = CL.Mlp(params=_params(8), in_scale=np.full(5, 300.0, np.float32), out_scale=0.002)
    m = dev(I.random_discs_mask(W, H, 2, 3.0, 5.0, 13))
    f0 = dev(I.perturbed_state(W, H, 14, amp=0.02))
    outs = []
    for storage in (SV.STORE_F32, SV.STORE_F16DEV):
        S = SV.Solver(W, H, storage=storage, collision=SV.COLL_MRT, closure=SV.CLOSURE_MLP, ref_clamps=0,
                      mlp=net.packed().data_ptr())
        a = S.new_state()
        SV.convert_state(f0, SV.STORE_F32, a, storage)
        b = a.clone()
        which = S.run(a, b, m, n, 2)
        r = torch.empty((9, H, W), device="cuda")
        SV.convert_state(b if which else a, storage, r, SV.STORE_F32)
        outs.append(host(r))
    assert rel_l2(outs[1], outs[0]) < 2e-3


def test_packed_block_for_another_activation_is_flagged():
    """A block packed for ReLU run as LBM_CLOSURE_MLP_SILU (or the reverse) sets
    bit 1 of the device error word; the matching pair leaves it clear."""
    W, H = 256, 64
    m = dev(I.random_discs_mask(W, H, 2, 3.0, 5.0, 13))
    f0 = I.perturbed_state(W, H, 14, amp=0.02)
    relu_net = CL.Mlp(params=_params(8), in_scale=np.full(5, 300.0, np.float32), out_scale=0.002, act="relu")
    for closure, want in ((SV.CLOSURE_MLP_SILU, 2), (SV.CLOSURE_MLP, 0)):
        SV.device_error_flags(clear=True)
        S = SV.Solver(W, H, collision=SV.COLL_MRT, closure=closure, ref_clamps=0, mlp=relu_net.packed().data_ptr())
        a, b = dev(f0), dev(f0)
        S.run(a, b, m, 4, 2)
        assert SV.device_error_flags(clear=True) & 2 == want
        S.close()
