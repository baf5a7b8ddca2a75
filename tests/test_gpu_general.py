"""GPU tests of the general solver (lbm_create / lbm_run and diagnostics)
against the general-solver oracle.

Tolerances: FP32 storage, relative L2 <= 1e-5 on the populations and on u, v,
rho of the last step (helpers.REL_TOL).  16-bit deviation storage is compared
with the FP64 oracle and its error is printed and bounded (see
test_storage_formats_error)."""
import os

import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, dev, host, rel_l2
from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu

BCS = {"wall": SV.BC_WALL, "periodic": SV.BC_PERIODIC, "zouhe": SV.BC_ZOUHE, "zouhe_ramp": SV.BC_ZOUHE_RAMP,
       "outflow": SV.BC_OUTFLOW}


def make(W, H, storage=SV.STORE_F32, collision="mrt", closure="smag", s_nu=1.8, s_e=1.1, s_eps=1.1, s_q=1.1,
         cs=0.2, bc_left="zouhe_ramp", bc_right="outflow", bc_y="wall", u_in=0.1, u_lid=0.0, ref_clamps=True):
    """A Solver and the oracle with the same parameters."""
    S = SV.Solver(W, H, storage=storage, collision=SV.COLL_MRT if collision == "mrt" else SV.COLL_BGK,
                  closure=SV.CLOSURE_SMAG if closure == "smag" else SV.CLOSURE_NONE, s_nu=s_nu, s_e=s_e, s_eps=s_eps,
                  s_q=s_q, cs_smag=cs, bc_left=BCS[bc_left], bc_right=BCS[bc_right], bc_y=BCS[bc_y], u_in=u_in,
                  u_lid=u_lid, ref_clamps=int(ref_clamps))
    G = O.General(W, H, collision=collision, closure=closure, s_nu=s_nu, s_e=s_e, s_eps=s_eps, s_q=s_q, cs=cs,
                  bc_left=bc_left, bc_right=bc_right, bc_y=bc_y, u_in=u_in, u_lid=u_lid, ref_clamps=ref_clamps)
    return S, G


CASES = {
    # the channel-past-a-cylinder physics of the bench workload
    "mrt_smag_clamps_ramp": (dict(cs=0.1, u_in=0.05, s_nu=1.0 / 0.50192), "discs"),
    "mrt_smag_flat_inlet": (dict(cs=0.1, u_in=0.05, s_nu=1.9, bc_left="zouhe", ref_clamps=False), "discs"),
    "cavity_lid": (dict(closure="none", bc_left="wall", bc_right="wall", u_lid=0.1, ref_clamps=False, s_e=1.1,
                        s_eps=1.0, s_q=1.2, s_nu=1.7), "cavity"),
    "bgk_periodic": (dict(collision="bgk", closure="none", bc_left="periodic", bc_right="periodic",
                          bc_y="periodic", ref_clamps=False, s_nu=1.5), "open"),
    "mrt_periodic_y_channel": (dict(closure="smag", cs=0.1, bc_y="periodic", ref_clamps=False, s_nu=1.8,
                                    u_in=0.04), "discs_open_y"),
}


def case_inputs(kind, W, H, seed=1):
    if kind == "discs":
        m = I.random_discs_mask(W, H, 3, 3.0, 6.0, seed)  # LBM_MASK_OBSTACLE discs
    elif kind == "cavity":
        m = I.cavity_mask(W, H)
    elif kind == "open":
        m = np.zeros((H, W), np.uint8)
    else:
        m = I.random_discs_mask(W, H, 2, 3.0, 5.0, seed)
        m[0, :] = 0
        m[H - 1, :] = 0
    f0 = I.perturbed_state(W, H, seed + 7, amp=0.02)
    return m, f0


@pytest.mark.parametrize("T", [1, 2, 3, 4, 5, 6, 8])
@pytest.mark.parametrize("W,H", [(130, 66), (136, 66), (256, 96)])  # 136: rows padded for the TMA mask map
@pytest.mark.parametrize("name", list(CASES))
def test_general_vs_oracle(name, W, H, T):
    kw, kind = CASES[name]
    S, G = make(W, H, **kw)
    m, f0 = case_inputs(kind, W, H)
    n = 9
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    which = S.run(a, b, dev(m), n, T, *mac)
    out = host(b if which else a)
    ref, rmac = G.run(m, f0, n)
    assert rel_l2(out, ref) < REL_TOL
    upd = m == 0
    for g_, r_ in zip(mac, rmac):
        assert rel_l2(host(g_)[upd], r_[upd]) < REL_TOL


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
def test_width_not_multiple_of_16_runs_padded_mask_rows(storage):
    """A width whose planes suit the register wavefront but whose mask rows do not
    (136 columns): lbm_run copies the mask into 16-byte aligned rows and runs the
    register wavefront, through the cached launch graphs (40 steps at T = 2); the
    result equals the oracle's and the caller's mask is left as it was."""
    W, H, n = 136, 66, 40
    kw, kind = CASES["mrt_smag_clamps_ramp"]
    S, G = make(W, H, storage=storage, **kw)
    m, f0 = case_inputs(kind, W, H)
    a = S.new_state()
    SV.convert_state(dev(f0), SV.STORE_F32, a, storage)
    b = a.clone()
    dm = dev(m)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    for _ in range(2):  # the second call replays the captured pair
        which = S.run(a, b, dm, n, 2, *mac)
        if which:
            a, b = b, a
    out = torch.empty((9, H, W), device="cuda")
    SV.convert_state(a, storage, out, SV.STORE_F32)
    ref, _ = G.run(m, f0, 2 * n)
    tol = REL_TOL if storage == SV.STORE_F32 else 2e-3
    assert rel_l2(host(out), ref) < tol
    assert np.array_equal(host(dm), m)
    S.close()


def test_equilibrium_init_matches_host():
    W, H = 96, 40
    S, _ = make(W, H)
    rng = np.random.default_rng(3)
    rho = (1 + 0.01 * rng.standard_normal((H, W))).astype(np.float32)
    ux = (0.05 * rng.standard_normal((H, W))).astype(np.float32)
    uy = (0.05 * rng.standard_normal((H, W))).astype(np.float32)
    f = S.new_state()
    S.init_equilibrium(f, dev(rho), dev(ux), dev(uy))
    want = I.equilibrium(rho, ux, uy)
    np.testing.assert_allclose(host(f), want, rtol=2e-6, atol=1e-7)


def test_diag_fp64_matches_host_and_is_deterministic():
    W, H = 300, 170
    S, _ = make(W, H)
    m, f0 = case_inputs("discs", W, H)
    f = dev(f0)
    d1 = host(S.diag(f, dev(m)))
    d2 = host(S.diag(f, dev(m)))
    assert np.array_equal(d1, d2)
    fl = m == 0
    f64 = f0.astype(np.float64)
    want = [f64[:, fl].sum(), (f64 * I.CX[:, None, None])[:, fl].sum(), (f64 * I.CY[:, None, None])[:, fl].sum()]
    np.testing.assert_allclose(d1, want, rtol=1e-12, atol=1e-9)


def test_mass_conservation_periodic_box():
    W, H = 128, 64
    S, _ = make(W, H, collision="bgk", closure="none", bc_left="periodic", bc_right="periodic", bc_y="periodic",
                ref_clamps=False, s_nu=1.6)
    m = np.zeros((H, W), np.uint8)
    _, f0 = case_inputs("open", W, H)
    a, b = dev(f0), dev(f0)
    mm = dev(m)
    d0 = host(S.diag(a, mm))
    which = S.run(a, b, mm, 400, 4)
    d1 = host(S.diag(b if which else a, mm))
    assert abs(d1[0] - d0[0]) < 2e-5 * d0[0]  # FP32 rounding drift over 400 steps; a leak would be O(1e-2)
    assert abs(d1[1] - d0[1]) < 2e-5 * d0[0] and abs(d1[2] - d0[2]) < 2e-5 * d0[0]


def test_forces_match_host_momentum_exchange():
    W, H = 200, 80
    S, _ = make(W, H, cs=0.1, u_in=0.05)
    m = I.cylinder_mask(W, H, 60, 40, 20)  # LBM_MASK_OBSTACLE
    f0 = I.perturbed_state(W, H, 11, amp=0.02)
    a, b = dev(f0), dev(f0)
    which = S.run(a, b, dev(m), 20, 4)
    f = b if which else a
    got = host(S.forces(f, dev(m)))
    fh = host(f).astype(np.float64)
    fx = fy = 0.0
    fl = m == 0
    for q in range(1, 9):
        nb = np.zeros_like(fl)
        cx, cy = int(I.CX[q]), int(I.CY[q])
        ys, xs = np.nonzero(fl)
        nx, ny = xs + cx, ys + cy
        ok = (nx >= 0) & (nx < W) & (ny >= 0) & (ny < H)
        ys, xs, nx, ny = ys[ok], xs[ok], nx[ok], ny[ok]
        hit = m[ny, nx] == I.OBSTACLE
        fx += 2 * cx * fh[q, ys[hit], xs[hit]].sum()
        fy += 2 * cy * fh[q, ys[hit], xs[hit]].sum()
    np.testing.assert_allclose(got, [fx, fy], rtol=1e-10, atol=1e-12)
    assert got[0] > 0  # the flow pushes the cylinder downstream


@pytest.mark.parametrize("storage", [SV.STORE_F16DEV, SV.STORE_BF16DEV])
def test_convert_state_round_trip(storage):
    W, H = 64, 32
    _, f0 = case_inputs("open", W, H)
    f = dev(f0)
    half = torch.empty(f.shape, dtype=torch.float16 if storage == SV.STORE_F16DEV else torch.bfloat16, device="cuda")
    back = torch.empty_like(f)
    SV.convert_state(f, SV.STORE_F32, half, storage)
    SV.convert_state(half, storage, back, SV.STORE_F32)
    w = I.WEIGHTS[:, None, None]
    dev_ = np.abs(f0 - w).max()
    tol = (2 ** -11 if storage == SV.STORE_F16DEV else 2 ** -8) * dev_ * 1.01
    assert np.abs(host(back) - f0).max() <= tol


def test_storage_formats_error():
    """FP16 / BF16 deviation storage against the FP64 oracle: relative L2 error of
    the velocity field after 200 steps of a channel flow past discs."""
    W, H = 256, 96
    kw = dict(cs=0.1, u_in=0.05, s_nu=1.9, ref_clamps=True)
    m, f0 = case_inputs("discs", W, H, seed=5)
    _, G = make(W, H, **kw)
    ref, rmac = G.run(m, f0.astype(np.float64), 200)
    uref = np.stack(rmac[:2])
    errs = {}
    for storage, tdt, bound in ((SV.STORE_F32, torch.float32, 1e-5), (SV.STORE_F16DEV, torch.float16, 5e-3),
                                (SV.STORE_BF16DEV, torch.bfloat16, 5e-2)):
        for T in (1, 4):
            S, _ = make(W, H, storage=storage, **kw)
            f32 = dev(f0)
            a = torch.empty(f32.shape, dtype=tdt, device="cuda")
            b = torch.empty_like(a)
            SV.convert_state(f32, SV.STORE_F32, a, storage)
            b.copy_(a)
            mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
            S.run(a, b, dev(m), 200, T, *mac)
            u = np.stack([host(mac[0]), host(mac[1])]).astype(np.float64)
            fl = m == 0
            err = rel_l2(u[:, fl], uref[:, fl])
            errs[f"storage{storage}_T{T}"] = err
            assert err < bound, (storage, T, err)
    print("velocity rel L2 vs FP64 oracle after 200 steps:", errs)


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
@pytest.mark.parametrize("T", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("name", ["mrt_smag_clamps_ramp", "cavity_lid", "mrt_periodic_y_channel"])
def test_register_wavefront_matches_smem_wavefront(name, T, storage):
    """The register wavefront kernel (TMA-aligned planes; 600 columns, so the mask
    rows go through the padded copy) against the shared-memory wavefront kernel
    (LBM_KERNEL=wave) and the oracle, on a domain of several windows and row chunks."""
    if name == "cavity_lid" and storage != SV.STORE_F32:
        pytest.skip("the moving-wall variant is built for FP32 storage only")
    W, H = 600, 264
    kw, kind = CASES[name]
    m, f0 = case_inputs(kind, W, H, seed=3)
    tdt = {SV.STORE_F32: torch.float32, SV.STORE_F16DEV: torch.float16}[storage]
    n = 2 * T + 1
    outs = []
    for kernel in ("", "wave"):
        os.environ["LBM_KERNEL"] = kernel
        try:
            S, G = make(W, H, storage=storage, **kw)
            a = torch.empty((9, H, W), dtype=tdt, device="cuda")
            SV.convert_state(dev(f0), SV.STORE_F32, a, storage)
            b = a.clone()
            mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
            which = S.run(a, b, dev(m), n, T, *mac)
            f32 = torch.empty((9, H, W), dtype=torch.float32, device="cuda")
            SV.convert_state(b if which else a, storage, f32, SV.STORE_F32)
            outs.append((host(f32), [host(x) for x in mac]))
        finally:
            os.environ.pop("LBM_KERNEL", None)
    (fr, mr), (fw, mw) = outs
    # same arithmetic in two kernels: a few ulps (of the storage format)
    assert rel_l2(fr, fw) < (1e-6 if storage == SV.STORE_F32 else REL_TOL)
    upd = m == 0
    for g_, w_ in zip(mr, mw):  # u, v are small: their relative error is a few times larger
        assert rel_l2(g_[upd], w_[upd]) < (5e-6 if storage == SV.STORE_F32 else 1e-4)
    if storage == SV.STORE_F32:
        ref, rmac = G.run(m, f0, n)
        assert rel_l2(fr, ref) < REL_TOL
        for g_, r_ in zip(mr, rmac):
            assert rel_l2(g_[upd], r_[upd]) < REL_TOL


def test_checked_run_reports_a_non_finite_state():
    """Failure detection by fault injection on the host: a NaN written into one
    fluid cell's populations is reported by the first check after it (an
    FP64 reduction of mass and momentum), and a clean run passes every check.
    (Without the reference clamps: fminf / fmaxf return the non-NaN operand, so
    the clamps replace a NaN population by a bound.)"""
    W, H = 256, 96
    kw, kind = CASES["mrt_smag_flat_inlet"]
    S, _ = make(W, H, **kw)
    m, f0 = case_inputs(kind, W, H)
    a, b = dev(f0), dev(f0)
    md = dev(m)
    which = S.run_checked(a, b, md, 40, T=2, check_every=10)
    assert torch.isfinite(b if which else a).all()
    a, b = dev(f0), dev(f0)
    ys, xs = np.nonzero(m == 0)
    a[3, ys[len(ys) // 2], xs[len(xs) // 2]] = float("nan")
    with pytest.raises(FloatingPointError, match="steps 1..10"):
        S.run_checked(a, b, md, 40, T=2, check_every=10)
