"""Parity at the full sizes of the benchmark configurations.

* The 4096 x 1024 cylinder channel (D = 128 at (1024, 512), MRT + Smagorinsky
  Cs = 0.1, Zou-He u = 0.05 with the ramp, nu = 6.4e-4, clamps on): the oracle
  runs 24 steps of the whole domain in a few seconds, so the populations and
  u, v, rho of every depth T = 1 .. 8 are compared with it (relative L2 <= 1e-5,
  FP32), from a perturbed state that makes every cell non-trivial.
* The 8192 x 2048 channel (D = 256 at (2048, 1024)) with FP32, FP16-deviation
  and BF16-deviation storage against the FP64 oracle (velocity relative L2
  <= 1e-5 / 5e-3 / 5e-2), and its FP64 mass and momentum sums against the same
  sums taken on the host.
* Longer runs at full size through properties that do not depend on the size:
  every depth gives the same state after 480 steps (the kernels differ only in
  rounding); a flat-inlet channel with a cylinder centred between the walls
  stays mirror-symmetric; a periodic 1024^2 box of decaying turbulence keeps its
  mass and momentum; a periodic box shifted by whole columns and rows gives the
  shifted result bit for bit.
* The 256-domain batch (sizes U[64, 1024]^2): every domain against the oracle
  (FP32), and the benchmark's FP16 batch against one launch per domain.
* The largest domain: 268 M cells, where plane offsets pass 2^31 elements."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, dev, host, rel_l2
from lbm_b200 import init as I
from lbm_b200 import solver as SV
from lbm_b200 import spectral as SP

pytestmark = pytest.mark.gpu

TAU = 0.50192
CHANNEL = dict(cs=0.1, u_in=0.05, s_nu=1.0 / TAU)


def _solver(W, H, storage=SV.STORE_F32, **kw):
    k = dict(CHANNEL)
    k.update(kw)
    return SV.Solver(W, H, storage=storage, cs_smag=k.pop("cs"), **k)


@pytest.fixture(scope="module")
def channel_4096():
    W, H, n = 4096, 1024, 24
    m = I.cylinder_mask(W, H, 1024, 512, 128, value=I.OBSTACLE)
    f0 = I.perturbed_state(W, H, 11, amp=0.02)
    G = O.General(W, H, **CHANNEL)
    ref, rmac = G.run(m, f0, n)
    return W, H, n, m, f0, ref, rmac


@pytest.mark.parametrize("T", [1, 2, 3, 4, 6, 8])
def test_channel_4096x1024_vs_oracle(channel_4096, T):
    W, H, n, m, f0, ref, rmac = channel_4096
    S = _solver(W, H)
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    which = S.run(a, b, dev(m), n, T, *mac)
    assert rel_l2(host(b if which else a), ref) < REL_TOL
    upd = m == 0
    for g_, r_ in zip(mac, rmac):
        assert rel_l2(host(g_)[upd], r_[upd]) < REL_TOL
    S.close()


def test_channel_8192x2048_storage_formats_vs_fp64_oracle():
    W, H, n = 8192, 2048, 8
    m = I.cylinder_mask(W, H, 2048, 1024, 256, value=I.OBSTACLE)
    f0 = I.perturbed_state(W, H, 13, amp=0.02)
    G = O.General(W, H, **CHANNEL)
    _, rmac = G.run(m, f0.astype(np.float64), n)
    fl = m == 0
    uref = np.stack(rmac[:2])[:, fl]
    mm = dev(m)
    errs = {}
    for storage, tdt, bound in ((SV.STORE_F32, torch.float32, REL_TOL), (SV.STORE_F16DEV, torch.float16, 5e-3),
                                (SV.STORE_BF16DEV, torch.bfloat16, 5e-2)):
        S = _solver(W, H, storage=storage)
        a = torch.empty((9, H, W), dtype=tdt, device="cuda")
        SV.convert_state(dev(f0), SV.STORE_F32, a, storage)
        b = a.clone()
        mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
        which = S.run(a, b, mm, n, 2, *mac)
        u = np.stack([host(mac[0]), host(mac[1])])[:, fl]
        errs[storage] = rel_l2(u, uref)
        assert errs[storage] < bound, (storage, errs[storage])
        if storage == SV.STORE_F32:
            f = b if which else a
            d = host(S.diag(f, mm))
            f64 = host(f).astype(np.float64)
            want = [f64[:, fl].sum(), (f64 * I.CX[:, None, None])[:, fl].sum(),
                    (f64 * I.CY[:, None, None])[:, fl].sum()]
            np.testing.assert_allclose(d, want, rtol=1e-11, atol=1e-7)
        S.close()
        del a, b, mac
        torch.cuda.empty_cache()
    print("8192x2048 velocity rel L2 vs FP64 oracle after", n, "steps:", errs)


def test_channel_4096x1024_depths_agree_after_480_steps():
    W, H, n = 4096, 1024, 480
    m = dev(I.cylinder_mask(W, H, 1024, 512, 128, value=I.OBSTACLE))
    f0 = dev(I.channel_state(W, H, u0=0.0, noise=1e-4, seed=0))
    S = _solver(W, H)
    out = {}
    for T in (1, 2, 3, 4, 6, 8):
        a, b = f0.clone(), f0.clone()
        which = S.run(a, b, m, n, T)
        out[T] = (b if which else a).clone()
        del a, b
    base = out[1].double()
    for T, f in out.items():
        err = (torch.linalg.vector_norm(f.double() - base) / torch.linalg.vector_norm(base)).item()
        assert err < REL_TOL, (T, err)
    S.close()


def test_flat_inlet_channel_stays_mirror_symmetric():
    """Cylinder centred between the walls (cy = (H - 1) / 2), uniform inlet: the
    field stays symmetric about the centre line (u_x even, u_y odd) up to
    rounding, which the mirrored cells accumulate in a different order."""
    W, H, n = 4096, 1024, 600
    m = I.cylinder_mask(W, H, 1024, (H - 1) / 2.0, 128, value=I.OBSTACLE)
    assert np.array_equal(m, m[::-1])
    S = _solver(W, H, bc_left=SV.BC_ZOUHE)
    a = dev(I.channel_state(W, H, u0=0.05))
    b = a.clone()
    mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    S.run(a, b, dev(m), n, 2, *mac)
    ux, uy = host(mac[0]).astype(np.float64), host(mac[1]).astype(np.float64)
    fl = m == 0
    scale = np.linalg.norm(ux[fl])
    ex = np.linalg.norm((ux - ux[::-1])[fl]) / scale
    ey = np.linalg.norm((uy + uy[::-1])[fl]) / scale
    assert np.linalg.norm(uy[fl]) > 1e-3 * scale  # the cylinder deflects the flow
    assert ex < 1e-5 and ey < 1e-5, (ex, ey)
    S.close()


def _periodic_solver(N):
    return SV.Solver(N, N, collision=SV.COLL_MRT, closure=SV.CLOSURE_SMAG, cs_smag=0.1, s_nu=1.0 / (3 * 5e-4 + 0.5),
                     s_e=1.64, s_eps=1.54, s_q=1.9, bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC,
                     bc_y=SV.BC_PERIODIC, ref_clamps=0)


def test_periodic_turbulence_1024_conserves_mass_and_momentum():
    N, n = 1024, 2000
    S = _periodic_solver(N)
    m = dev(np.zeros((N, N), np.uint8))
    a = dev(SP.turbulence_state(N, seed=3))
    b = a.clone()
    d0 = host(S.diag(a, m))
    which = S.run(a, b, m, n, 2)
    d1 = host(S.diag(b if which else a, m))
    drift = np.abs(d1 - d0) / d0[0]
    print("mass / momentum drift after", n, "steps:", drift)
    assert drift[0] < 1e-8 and drift[1] < 1e-8 and drift[2] < 1e-8, drift  # measured 5e-10 / 8e-12 / 6e-12
    S.close()


def test_periodic_box_is_translation_equivariant():
    """Shifting the initial state by whole columns and rows shifts the result
    bit for bit (the same arithmetic runs at every cell, wrapped edges included)."""
    N, n, dx, dy = 1024, 200, 64, 37
    S = _periodic_solver(N)
    m = dev(np.zeros((N, N), np.uint8))
    f0 = SP.turbulence_state(N, seed=4)
    a = dev(f0)
    b = a.clone()
    which = S.run(a, b, m, n, 2)
    r0 = host(b if which else a)
    a = dev(np.roll(f0, (dy, dx), axis=(1, 2)))
    b = a.clone()
    which = S.run(a, b, m, n, 2)
    r1 = host(b if which else a)
    err = rel_l2(r1, np.roll(r0, (dy, dx), axis=(1, 2)))
    assert err == 0.0, err
    S.close()


def _batch_256(storage, tdt, perturbed):
    """The 256-domain batch configuration: Nx, Ny ~ U[64, 1024], 1-4 discs of
    radius 4-32, inlet u ~ U[0.02, 0.08] (seeded as the benchmark builds it)."""
    rng = np.random.default_rng(1234)
    doms, hosts = [], []
    for i in range(256):
        w, h = int(rng.integers(64, 1025)), int(rng.integers(64, 1025))
        m = I.random_discs_mask(w, h, int(rng.integers(1, 5)), 4.0, min(32.0, h / 4), 5000 + i)
        u_in = float(rng.uniform(0.02, 0.08))
        pitch = (w + 15) // 16 * 16
        mk = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
        mk[:, :w] = dev(m)
        f0 = I.perturbed_state(w, h, 7000 + i, amp=0.02) if perturbed else None
        fa = torch.zeros((9, h, pitch), dtype=tdt, device="cuda")
        if perturbed:
            fa[:, :, :w] = dev(f0)
        doms.append(dict(W=w, H=h, pitch=pitch, mask_pitch=pitch, f_a=fa, f_b=fa.clone(), mask=mk, u_in=u_in))
        hosts.append((m, f0, u_in))
    return doms, hosts


def test_batch_of_256_domains_vs_oracle():
    """Every domain of the full 256-domain batch (FP32 storage here, from
    perturbed states) against the oracle run of that domain alone."""
    from lbm_b200.batch import Batch

    doms, hosts = _batch_256(SV.STORE_F32, torch.float32, True)
    B = Batch(doms, storage=SV.STORE_F32, cs_smag=0.1, s_nu=1.0 / TAU)
    n = 9
    which = B.run(n, 4)
    worst = 0.0
    for d, (m, f0, u_in) in zip(doms, hosts):
        W = d["W"]
        out = host((d["f_b"] if which else d["f_a"])[:, :, :W].contiguous())
        G = O.General(W, d["H"], cs=0.1, s_nu=1.0 / TAU, u_in=u_in)
        ref, _ = G.run(m, f0, n)
        worst = max(worst, rel_l2(out, ref))
    assert worst < REL_TOL, worst


def test_batch_of_256_domains_fp16_equals_separate_launches():
    """The benchmark's batch exactly (FP16 deviations, fluid at rest): one
    launch per T steps for all domains equals one launch per domain."""
    from lbm_b200.batch import Batch

    doms1, _ = _batch_256(SV.STORE_F16DEV, torch.float16, False)
    doms2, _ = _batch_256(SV.STORE_F16DEV, torch.float16, False)
    B1 = Batch(doms1, storage=SV.STORE_F16DEV, cs_smag=0.1, s_nu=1.0 / TAU)
    B2 = Batch(doms2, storage=SV.STORE_F16DEV, cs_smag=0.1, s_nu=1.0 / TAU)
    w1 = B1.run(40, 4)
    w2 = B2.run_separate(40, 4)
    assert w1 == w2
    wts = I.WEIGHTS[:, None, None].astype(np.float32)
    worst = 0.0
    for d1, d2 in zip(doms1, doms2):
        W = d1["W"]
        a = host((d1["f_b"] if w1 else d1["f_a"])[:, :, :W].float()) + wts
        b = host((d2["f_b"] if w2 else d2["f_a"])[:, :, :W].float()) + wts
        worst = max(worst, rel_l2(a, b))
    assert worst < REL_TOL, worst


@pytest.mark.parametrize("storage,T", [(SV.STORE_F32, 1), (SV.STORE_F32, 2), (SV.STORE_F32, 4),
                                       (SV.STORE_F16DEV, 2), (SV.STORE_F32, "inplace")])
def test_largest_domain_repeats_the_small_result(storage, T):
    """A 4096 x 65536 channel (268 M cells: plane offsets pass 2^31 elements),
    periodic in y, built as 64 copies of a 4096 x 1024 channel stacked in y.
    Every copy sees the neighbourhood of the small periodic domain, so after 8
    steps each copy equals the small domain's result bit for bit."""
    W, h, reps, n = 4096, 1024, 64, 8
    m = I.random_discs_mask(W, h, 6, 8.0, 40.0, 21)
    m[0, :] = 0
    m[h - 1, :] = 0
    kw = dict(bc_y=SV.BC_PERIODIC, bc_left=SV.BC_ZOUHE, ref_clamps=0)  # flat inlet: no y-dependent ramp
    tdt = torch.float32 if storage == SV.STORE_F32 else torch.float16
    f0 = torch.empty((9, h, W), dtype=tdt, device="cuda")
    SV.convert_state(dev(I.perturbed_state(W, h, 23, amp=0.02)), SV.STORE_F32, f0, storage)

    def run(S, mask, a):
        if T == "inplace":
            S.run_inplace(a, mask, n)
            return a
        b = a.clone()
        which = S.run(a, b, mask, n, T)
        return b if which else a

    small = run(_solver(W, h, storage=storage, **kw), dev(m), f0.clone())
    S = _solver(W, h * reps, storage=storage, **kw)
    big = run(S, dev(np.tile(m, (reps, 1))), f0.repeat(1, reps, 1))
    torch.cuda.synchronize()
    assert torch.equal(big.view(9, reps, h, W), small.unsqueeze(1).expand(9, reps, h, W))
    S.close()
