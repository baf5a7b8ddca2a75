"""Learned-closure oracle checks on CPU: the numpy MLP's gradient against finite
differences, the oracle's MLP closure against a constant-viscosity MRT step, and
the a-priori training targets on analytic fields."""
import numpy as np
import pytest

import mlp_oracle as MO
import oracle as O
from lbm_b200 import closure as CL
from lbm_b200 import init as I


@pytest.mark.parametrize("act", ["relu", "silu"])
def test_oracle_gradient_matches_finite_differences(act):
    rng = np.random.default_rng(0)
    p = CL.init_params(3).astype(np.float64) + 0.05 * rng.standard_normal(MO.NPARAM)
    x = rng.standard_normal((40, 5))
    t = rng.random(40)
    w = rng.random(40) + 0.5
    _, g = MO.loss_grad(p, x, t, w, act=act)
    idx = rng.choice(MO.NPARAM, 60, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (MO.loss_grad(pp, x, t, w, act=act)[0] - MO.loss_grad(pm, x, t, w, act=act)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_oracle_mlp_closure_with_constant_output_is_plain_mrt():
    W, H = 40, 24
    p = np.zeros(MO.NPARAM, np.float32)
    p[MO.OB3] = 0.3  # nu_t = out_scale softplus(0.3) everywhere
    out_scale = 0.01
    O.set_mlp(p, np.ones(5, np.float32), out_scale)
    nu_t = out_scale * np.log1p(np.exp(0.3))
    s_nu = 1.8
    s_eff = 1.0 / (1.0 / s_nu + 3.0 * nu_t)
    m = I.random_discs_mask(W, H, 2, 2.0, 4.0, 1)
    f0 = I.perturbed_state(W, H, 2, amp=0.02).astype(np.float64)
    kw = dict(collision="mrt", bc_left="wall", bc_right="wall", bc_y="periodic", ref_clamps=False)
    a, _ = O.General(W, H, closure="mlp", s_nu=s_nu, **kw).run(m, f0, 5)
    b, _ = O.General(W, H, closure="none", s_nu=s_eff, **kw).run(m, f0, 5)
    assert np.abs(a - b).max() < 1e-10  # the two evaluate the rate 1 / (tau0 + 3 nu) differently


def test_training_targets_on_analytic_fields():
    # a pure shear u = U sin(2 pi y / L): no subgrid stress at the filter scale
    # of a smooth mode beyond the filter's own smoothing, targets stay >= 0
    N, f = 64, 4
    y = np.arange(N * f)[:, None] * np.ones((1, N * f))
    u = 0.05 * np.sin(2 * np.pi * y / (N * f))
    v = np.zeros_like(u)
    x, nu = CL.targets_and_features(u, v, np.ones_like(u), f, tau0=0.6, s_e=1.1)
    assert x.shape == (N * N, 5) and nu.shape == (N * N,)
    assert (nu >= 0).all() and np.isfinite(x).all()
    # n8 carries the shear: -(2/3) tau_eff S_xy with S_xy = dU/dy / 2
    assert np.abs(x[:, 1]).max() > 0 and np.abs(x[:, 0]).max() < 1e-9
    # the Smagorinsky viscosity of the same features is nonnegative and grows with |S|
    ns = CL.smagorinsky_nu(x, 0.1, 0.6)
    assert (ns >= 0).all() and np.corrcoef(ns, x[:, 3])[0, 1] > 0.99
