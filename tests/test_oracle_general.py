"""Known-answer tests of the general-solver oracle (CPU): invariants any correct
D2Q9 solver with these boundary rules must satisfy."""
import numpy as np

import oracle as O
from lbm_b200 import init as I


def test_equilibrium_moments_round_trip():
    rng = np.random.default_rng(0)
    rho = 1.0 + 0.05 * rng.standard_normal((8, 8))
    ux = 0.05 * rng.standard_normal((8, 8))
    uy = 0.05 * rng.standard_normal((8, 8))
    f = I.equilibrium(rho, ux, uy, dtype=np.float64)
    r = f.sum(0)
    np.testing.assert_allclose(r, rho, rtol=1e-12)
    np.testing.assert_allclose((f * I.CX[:, None, None]).sum(0) / r, ux, atol=1e-12)
    np.testing.assert_allclose((f * I.CY[:, None, None]).sum(0) / r, uy, atol=1e-12)


def test_rest_state_is_invariant():
    W, H = 24, 16
    m = np.zeros((H, W), np.uint8)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = 1
    f0 = I.equilibrium(np.ones((H, W)), np.zeros((H, W)), np.zeros((H, W)), dtype=np.float64)
    g = O.General(W, H, closure="smag", cs=0.1, bc_left="wall", bc_right="wall", ref_clamps=False, s_nu=1.9)
    f, _ = g.run(m, f0, 20)
    fl = m == 0
    np.testing.assert_allclose(f[:, fl], f0[:, fl], atol=1e-14)


def test_mass_conserved_in_periodic_box():
    W, H = 32, 24
    m = np.zeros((H, W), np.uint8)
    f0 = I.perturbed_state(W, H, 3, amp=0.03).astype(np.float64)
    for coll in ("bgk", "mrt"):
        g = O.General(W, H, collision=coll, closure="none", bc_left="periodic", bc_right="periodic",
                      bc_y="periodic", ref_clamps=False, s_nu=1.6)
        f, _ = g.run(m, f0, 40)
        assert abs(f.sum() - f0.sum()) < 1e-10 * f0.sum()
        # momentum is conserved too (no walls, no forcing)
        for c in (I.CX, I.CY):
            p0 = (f0 * c[:, None, None]).sum()
            p1 = (f * c[:, None, None]).sum()
            assert abs(p1 - p0) < 1e-10


def test_mrt_with_equal_rates_is_bgk():
    W, H = 20, 12
    m = np.zeros((H, W), np.uint8)
    f0 = I.perturbed_state(W, H, 5, amp=0.03).astype(np.float64)
    s = 1.3
    kw = dict(closure="none", bc_left="periodic", bc_right="periodic", bc_y="periodic", ref_clamps=False, s_nu=s)
    fm, _ = O.General(W, H, collision="mrt", s_e=s, s_eps=s, s_q=s, **kw).run(m, f0, 5)
    fb, _ = O.General(W, H, collision="bgk", **kw).run(m, f0, 5)
    np.testing.assert_allclose(fm, fb, atol=1e-12)


def test_bounce_back_returns_a_pulse():
    """A single east-moving population next to an east wall comes back west."""
    W, H = 6, 3
    m = np.zeros((H, W), np.uint8)
    m[:, W - 1] = 1
    rest = I.equilibrium(np.ones((H, W)), np.zeros((H, W)), np.zeros((H, W)), dtype=np.float64)
    f0 = rest.copy()
    f0[1, 1, W - 2] += 0.01  # extra post-collision population moving east, next to the wall
    g = O.General(W, H, collision="bgk", closure="none", bc_left="periodic", bc_right="periodic", bc_y="periodic",
                  ref_clamps=False, s_nu=1e-12)  # (almost) no collision: pure streaming
    f1, _ = g.step(m, f0, f0.copy())
    d = f1 - rest
    assert abs(d[3, 1, W - 2] - 0.01) < 1e-9  # came back west in the same cell
    assert abs(d[:, m == 0].sum() - 0.01) < 1e-9 and abs(d[1, m == 0]).max() < 1e-9


def test_zou_he_inlet_imposes_velocity():
    W, H = 40, 30
    m = I.channel_mask(W, H)
    f0 = I.channel_state(W, H, dtype=np.float64)
    for bc, ramp in (("zouhe", False), ("zouhe_ramp", True)):
        g = O.General(W, H, collision="mrt", closure="smag", cs=0.1, bc_left=bc, u_in=0.05, ref_clamps=False)
        _, (ux, uy, _) = g.run(m, f0, 3)
        y = np.arange(1, H - 1)
        d = np.minimum(y, H - 1 - y).astype(np.float64)
        want = 0.05 * np.where(d < 50, 0.5 * (1 - np.cos(np.float32(3.14159) * d / 50)), 1.0) if ramp else 0.05
        np.testing.assert_allclose(ux[1:H - 1, 0], want, rtol=1e-6)
        assert np.all(uy[1:H - 1, 0] == 0)


def test_moving_lid_drives_the_cavity():
    W, H = 32, 32
    m = I.cavity_mask(W, H)
    f0 = I.equilibrium(np.ones((H, W)), np.zeros((H, W)), np.zeros((H, W)), dtype=np.float64)
    g = O.General(W, H, closure="none", bc_left="wall", bc_right="wall", u_lid=0.1, ref_clamps=False, s_e=1.1,
                  s_eps=1.0, s_q=1.2, s_nu=1.7)
    f, (ux, _, _) = g.run(m, f0, 200)
    assert ux[H - 2, W // 2] > 0.03  # the row under the lid follows it
    assert ux[H // 4, W // 2] < 0.0  # return flow lower down
    # mass is conserved by half-way bounce-back (moving wall with rho_w = 1 adds
    # zero net mass for a wall parallel to itself)
    assert abs(f[:, m == 0].sum() - f0[:, m == 0].sum()) < 1e-9 * f0.sum()


def test_general_reduces_to_core4():
    """With the lbm_core4.cu constants and the driver's mask conventions the
    general rules give the reference step."""
    W, H = 48, 32
    m = I.random_discs_mask(W, H, 2, 3.0, 5.0, 4, value=1)
    f0 = I.perturbed_state(W, H, 6).astype(np.float64)
    g = O.General(W, H, collision="mrt", closure="smag", cs=0.2, s_nu=1.8, u_in=0.1)
    fg, mg = g.run(m, f0, 4)
    fc, mc = O.core4_run(m, f0, 4, tau_inv=1.8, u_in=0.1)
    np.testing.assert_allclose(fg, fc, atol=1e-12)
    for a, b in zip(mg, mc):
        np.testing.assert_allclose(a, b, atol=1e-12)


def test_poiseuille_profile_is_the_parabola():
    """Channel with a flat Zou-He inlet, an outflow and half-way bounce-back walls
    (fluid rows 1 .. H-2, walls at y = 1/2 and y = H - 3/2): downstream of the
    inlet the velocity profile has the shape of the parabola (y - 1/2)(H - 3/2 - y)
    of width L = H - 2 (max / mean = 3/2).  The shape, not the level: with a
    velocity inlet and a zero-gradient outlet (the reference's boundary pair) the
    channel has no pressure reference, so the density, and with it the mean speed
    at a given x, drifts."""
    W, H, u0, nu = 96, 18, 0.04, 0.1
    g = O.General(W, H, collision="mrt", closure="none", s_nu=1.0 / (3 * nu + 0.5), s_e=1.1, s_eps=1.1, s_q=1.1,
                  bc_left="zouhe", bc_right="outflow", bc_y="wall", u_in=u0, ref_clamps=False)
    m = I.channel_mask(W, H)
    f0 = I.channel_state(W, H, u0=u0, dtype=np.float64)
    _, mac = g.run(m, f0, 3000)
    y = np.arange(1, H - 1, dtype=np.float64)
    shape = (y - 0.5) * (H - 1.5 - y)
    for x in (40, 70):
        u = np.asarray(mac[0])[1:H - 1, x]
        a = u / u.mean()
        b = shape / shape.mean()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 0.01, x
        assert abs(u.max() / u.mean() - 1.5) < 0.01
