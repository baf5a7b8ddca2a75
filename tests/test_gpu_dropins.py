"""GPU parity of the reference drop-ins (C-ABI, liblbm_b200.so) against the CPU
oracle on seeded inputs and against the reference's own kernels (oracle/_ref).

Tolerance: relative L2 error <= 1e-5 (helpers.REL_TOL) on u, v, rho and the
populations, FP32 with -use_fast_math on both GPU sides."""
import numpy as np
import pytest
import torch

import lbm_b200 as L
import oracle as O
from helpers import REL_TOL, away_from_outlet_corners, dev, host, ptr, ref_lib, rel_l2, stream, zeros
from lbm_b200 import init as I

pytestmark = pytest.mark.gpu

SIZES = [(64, 48), (130, 66), (256, 96)]  # 64/256: TMA path, 130: plain-load path


def _case(W, H, seed):
    mask = I.random_discs_mask(W, H, 3, 3.0, 7.0, seed, value=1)
    f0 = I.perturbed_state(W, H, seed + 10)
    return mask, f0


@pytest.mark.parametrize("W,H", SIZES)
def test_core4_step_vs_oracle(W, H):
    mask, f0 = _case(W, H, 1)
    m, a = dev(mask), dev(f0)
    b = a.clone()
    mac = [zeros(H, W) for _ in range(3)]
    ref_a, ref_b = f0.copy(), f0.copy()
    ref_mac = tuple(np.zeros((H, W), np.float32) for _ in range(3))
    for step in range(1, 13):
        L.core4_step(m, a, b, *mac, W, H, 1.8, 0.1)
        a, b = b, a
        O.core4_step(mask, ref_a, ref_b, ref_mac, tau_inv=1.8, u_in=0.1)
        ref_a, ref_b = ref_b, ref_a
        if step in (1, 2, 5, 12):
            assert rel_l2(host(a), ref_a) < REL_TOL, step
            for g, r in zip(mac, ref_mac):
                assert rel_l2(host(g), r) < REL_TOL, step


@pytest.mark.parametrize("T", [2, 3, 4, 5, 8])
@pytest.mark.parametrize("W,H", [(130, 66), (256, 96)])
def test_core4_run_blocked_equals_single_steps(W, H, T):
    """T steps fused in one launch reproduce single-step launches.  The arithmetic
    is the same; the compiler may contract different multiply-adds in different
    instantiations, so the bound is a few FP32 ulps rather than bit equality."""
    mask, f0 = _case(W, H, 2)
    m = dev(mask)
    n = 2 * T + 1
    a, b = dev(f0), dev(f0)
    mac = [zeros(H, W) for _ in range(3)]
    for _ in range(n):
        L.core4_step(m, a, b, *mac, W, H, 1.8, 0.1)
        a, b = b, a
    a2, b2 = dev(f0), dev(f0)
    mac2 = [zeros(H, W) for _ in range(3)]
    which = L.core4_run(m, a2, b2, *mac2, W, H, 1.8, 0.1, n, T)
    out = b2 if which else a2
    assert rel_l2(host(out), host(a)) < 1e-6
    assert np.abs(host(out) - host(a)).max() < 1e-5
    for g, r in zip(mac2, mac):
        assert rel_l2(host(g), host(r)) < REL_TOL


def _driver_case(W=2048, H=512):
    """The lbm_mine2.py set-up: Gaussian-pair u_x, rho = 1, channel with a disc."""
    mask = I.cylinder_mask(W, H, W // 4, H // 2, H // 8, value=1)
    ux = I.gaussian_pair_ux(W, H)
    f0 = I.equilibrium(np.ones((H, W)), ux, np.zeros((H, W)))
    return mask, f0


@pytest.mark.parametrize("W,H", [(2048, 512), (4096, 1024)])
def test_core4_vs_reference_kernel_driver_size(W, H):
    """The drivers' 2048 x 512 case, and the same set-up at 4096 x 1024 (a
    D = 128 disc at (1024, 512): the cylinder channel's geometry)."""
    lib = ref_lib("libref_core4.so")
    if lib is None:
        pytest.skip("oracle/_ref not built")
    mask, f0 = _driver_case(W, H)
    m = dev(mask)
    a, b = dev(f0), dev(f0)
    ra, rb = dev(f0), dev(f0)
    mac = [zeros(H, W) for _ in range(3)]
    rmac = [zeros(H, W) for _ in range(3)]
    for _ in range(50):
        L.core4_step(m, a, b, *mac, W, H, 1.8, 0.1)
        a, b = b, a
        assert lib.ref_core4_step(ptr(m), ptr(ra), ptr(rb), *[ptr(t) for t in rmac], W, H, 1.8, 0.1, 1.8,
                                  stream()) == 0
        ra, rb = rb, ra
    assert rel_l2(host(a), host(ra)) < REL_TOL
    for g, r in zip(mac, rmac):
        assert rel_l2(host(g), host(r)) < REL_TOL


@pytest.mark.parametrize("W,H", [(2048, 512), (4096, 1024)])
def test_core4_run_vs_reference_kernel_driver_size(W, H):
    """lbm_core4_run at T = 2 (the register wavefront with the packed two-cell
    collision in the reference's evaluation order) against the reference kernel
    stepped 50 times, at the drivers' size and the cylinder channel's."""
    lib = ref_lib("libref_core4.so")
    if lib is None:
        pytest.skip("oracle/_ref not built")
    mask, f0 = _driver_case(W, H)
    m = dev(mask)
    a, b = dev(f0), dev(f0)
    ra, rb = dev(f0), dev(f0)
    mac = [zeros(H, W) for _ in range(3)]
    rmac = [zeros(H, W) for _ in range(3)]
    which = L.core4_run(m, a, b, *mac, W, H, 1.8, 0.1, 50, 2)
    for _ in range(50):
        assert lib.ref_core4_step(ptr(m), ptr(ra), ptr(rb), *[ptr(t) for t in rmac], W, H, 1.8, 0.1, 1.8,
                                  stream()) == 0
        ra, rb = rb, ra
    assert rel_l2(host(b if which else a), host(ra)) < REL_TOL
    for g, r in zip(mac, rmac):
        assert rel_l2(host(g), host(r)) < REL_TOL


@pytest.mark.parametrize("W,H", SIZES)
def test_smemaa_vs_oracle(W, H):
    mask, f0 = _case(W, H, 3)
    m, a = dev(mask), dev(f0)
    b = a.clone()
    mac = [zeros(H, W) for _ in range(3)]
    ra, rb = f0.copy(), f0.copy()
    rmac = tuple(np.zeros((H, W), np.float32) for _ in range(3))
    for n in range(1, 4):
        L.smemaa_step(m, a, b, *mac, W, H, 1.7, 0.1, T=4)
        a, b = b, a
        O.smemaa_launch(mask, ra, rb, rmac, tau_inv=1.7, u_in=0.1, T=4)
        ra, rb = rb, ra
        assert rel_l2(host(a), ra) < REL_TOL, n
        for g, r in zip(mac, rmac):
            assert rel_l2(host(g), r) < REL_TOL, n


@pytest.mark.parametrize("T", [2, 4, 6, 8])
def test_smemaa_depths_vs_oracle(T):
    W, H = 130, 66
    mask, f0 = _case(W, H, 4)
    m, a = dev(mask), dev(f0)
    b = a.clone()
    mac = [zeros(H, W) for _ in range(3)]
    L.smemaa_step(m, a, b, *mac, W, H, 1.7, 0.1, T=T)
    rb, rmac = O.smemaa_launch(mask, f0, f0.copy(), None, tau_inv=1.7, u_in=0.1, T=T)
    assert rel_l2(host(b), rb) < REL_TOL
    for g, r in zip(mac, rmac):
        assert rel_l2(host(g), r) < REL_TOL


@pytest.mark.parametrize("T", [2, 4, 6, 8])
@pytest.mark.parametrize("W,H", SIZES)
def test_blocked_vs_oracle(W, H, T):
    """Our kernel defines every slot (initialised from f_now, like lbm_core_smemaa.cu),
    so it matches the oracle everywhere, corners included."""
    mask = I.random_discs_mask(W, H, 3, 3.0, 7.0, 5, value=1)
    f0 = I.perturbed_state(W, H, 15)
    m, a = dev(mask), dev(f0)
    b = a.clone()
    ra, rb = f0.copy(), f0.copy()
    for n in range(2):
        L.blocked_step(m, a, b, W, H, 1.0, 0.1, T=T)
        a, b = b, a
        O.policy_launch(mask, ra, rb, tau_inv=1.0, u_in=0.1, T=T)
        ra, rb = rb, ra
        assert rel_l2(host(a), ra) < REL_TOL
        assert rel_l2(host(b), rb) < REL_TOL
    mac = [zeros(H, W) for _ in range(3)]
    L.macro(a, *mac, m, W, H, 0.1)
    rmac = O.macro(ra, mask, u_in=0.1)
    for g, r in zip(mac, rmac):
        assert rel_l2(host(g), r) < REL_TOL


@pytest.mark.parametrize("W,H", [(2048, 512), (4096, 1024)])
@pytest.mark.parametrize("libname,kind", [("libref_smemaa.so", "smemaa"), ("libref_policy.so", "policy"),
                                          ("libref_endfused.so", "endfused")])
def test_blocked_vs_reference_kernel_driver_size(libname, kind, W, H):
    """At 4096 x 1024 (4.2 M cells) the drop-ins take the split launch (edge
    tiles beside the interior register wavefront)."""
    lib = ref_lib(libname)
    if lib is None:
        pytest.skip("oracle/_ref not built")
    mask, f0 = _driver_case(W, H)
    T = lib.ref_T()
    n = 8
    m = dev(mask)
    a, b = dev(f0), dev(f0)
    ra, rb = dev(f0), dev(f0)
    mac = [zeros(H, W) for _ in range(3)]
    rmac = [zeros(H, W) for _ in range(3)]
    tau = 1.7 if kind == "smemaa" else 1.0
    for _ in range(n):
        if kind == "smemaa":
            L.smemaa_step(m, a, b, *mac, W, H, tau, 0.1, T=T)
            assert lib.ref_smemaa_step(ptr(m), ptr(ra), ptr(rb), *[ptr(t) for t in rmac], W, H, tau, 0.1,
                                       stream()) == 0
        else:
            L.blocked_step(m, a, b, W, H, tau, 0.1, T=T)
            assert lib.ref_blocked_step(ptr(m), ptr(ra), ptr(rb), W, H, tau, 0.1, stream()) == 0
        a, b = b, a
        ra, rb = rb, ra
    # smemaa initialises every slot; policy/endfused do not at the outlet corners.
    ok = np.ones((H, W), bool) if kind == "smemaa" else away_from_outlet_corners(W, H, n * T + 2)
    assert rel_l2(host(a)[:, ok], host(ra)[:, ok]) < REL_TOL
    if kind != "smemaa":
        L.macro(a, *mac, m, W, H, 0.1)
        assert lib.ref_macro(ptr(ra), *[ptr(t) for t in rmac], ptr(m), W, H, 0.1, stream()) == 0
    for g, r in zip(mac, rmac):
        assert rel_l2(host(g)[ok], host(r)[ok]) < REL_TOL


def test_visualize_vs_oracle_and_reference():
    W, H = 96, 40
    rng = np.random.default_rng(8)
    mask = I.random_discs_mask(W, H, 2, 3.0, 6.0, 8, value=1)
    ux = (0.02 * rng.standard_normal((H, W))).astype(np.float32)
    uy = (0.02 * rng.standard_normal((H, W))).astype(np.float32)
    import torch

    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    L.visualize(dev(ux), dev(uy), None, img, dev(mask), W, H, 50.0)
    want = O.visualize(ux, uy, mask, 50.0)
    np.testing.assert_array_equal(host(img), want)
    lib = ref_lib("libref_core4.so")
    if lib is not None:
        rimg = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        keep = [dev(ux), dev(uy), dev(np.ones((H, W), np.float32)), rimg, dev(mask)]  # alive until the kernel ran
        assert lib.ref_visualize(*[ptr(t) for t in keep], W, H, 50.0, stream()) == 0
        np.testing.assert_array_equal(host(img), host(rimg))


def test_refcompat_module_shape():
    """The RawModule-shaped shim accepts the reference's (grid, block, args) call."""
    W, H = 128, 64
    mask, f0 = _case(W, H, 9)
    m, a = dev(mask), dev(f0)
    b = a.clone()
    mac = [zeros(H, W) for _ in range(3)]
    mod = L.RefCompatModule("core4")
    k = mod.get_function("fused_lbmkernel")
    k((64, 64), (32, 8), (m, a, b, *mac, np.int32(W), np.int32(H), np.float32(1.8), np.float32(0.1),
                          np.float32(1.8)))
    ref, rmac = O.core4_step(mask, f0, f0.copy(), tau_inv=1.8, u_in=0.1)
    assert rel_l2(host(b), ref) < REL_TOL
    pol = L.RefCompatModule("policy")
    assert pol.T == 6 and pol.get_function("macro_kernel") is not None


@pytest.mark.parametrize("kind", ["smemaa", "policy"])
@pytest.mark.parametrize("T", [2, 4, 6])
def test_split_launch_matches_tile_kernel(kind, T):
    """lbm_smemaa_step / lbm_blocked_step on TMA-aligned buffers run the AA tile
    kernel on the edge band and the register wavefront (pre-collision mode) inside;
    the result must equal the tile kernel everywhere (LBM_AA_SPLIT=0)."""
    import os

    W, H, n = 2048, 2048, 2  # the split runs on domains of at least 4 M cells
    m = I.random_discs_mask(W, H, 12, 3.0, 12.0, 21)
    f0 = I.perturbed_state(W, H, 22, amp=0.02)
    outs = []
    for split in ("1", "0"):
        os.environ["LBM_AA_SPLIT"] = split
        try:
            a, b = dev(f0), dev(f0)
            mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
            for _ in range(n):
                if kind == "smemaa":
                    L.smemaa_step(dev(m), a, b, *mac, W, H, 1.7, 0.1, T=T)
                else:
                    L.blocked_step(dev(m), a, b, W, H, 1.7, 0.1, T=T)
                a, b = b, a
            torch.cuda.synchronize()
            outs.append((host(a), [host(x) for x in mac]))
        finally:
            os.environ.pop("LBM_AA_SPLIT", None)
    (fs, ms), (ft, mt) = outs
    # the interior's packed two-cell collision rounds like the tile kernel's scalar
    # one up to the multiply-adds the compiler contracts: a few ulps (u, v are small,
    # so their relative error is a few times larger)
    assert rel_l2(fs, ft) < 1e-6
    if kind == "smemaa":
        for x, y in zip(ms, mt):
            assert rel_l2(x, y) < 5e-6


def test_split_launch_from_two_host_threads():
    """Two host threads run split AA launches at the same time, each on its own
    stream and its own state; each result must equal the unsplit tile kernel
    (LBM_AA_SPLIT=0) on the same inputs.  The split's side stream and fork/join
    events belong to the calling thread, so neither thread's edge-band kernel can
    wait on the other's stream."""
    import os
    import threading

    W, H, n, T = 2048, 2048, 6, 4
    cases = []
    for seed in (31, 32):
        m = I.random_discs_mask(W, H, 10, 3.0, 12.0, seed)
        cases.append((m, I.perturbed_state(W, H, seed + 5, amp=0.02)))
    os.environ["LBM_AA_SPLIT"] = "0"
    try:
        want = []
        for m, f0 in cases:
            a, b = dev(f0), dev(f0)
            mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
            for _ in range(n):
                L.smemaa_step(dev(m), a, b, *mac, W, H, 1.7, 0.1, T=T)
                a, b = b, a
            want.append(host(a))
    finally:
        os.environ.pop("LBM_AA_SPLIT", None)

    got, errors = [None, None], []

    def worker(k):
        try:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                m, f0 = cases[k]
                dm, a, b = dev(m), dev(f0), dev(f0)
                mac = [torch.zeros((H, W), device="cuda") for _ in range(3)]
                for _ in range(n):
                    L.smemaa_step(dm, a, b, *mac, W, H, 1.7, 0.1, T=T, stream=st.cuda_stream)
                    a, b = b, a
            st.synchronize()
            got[k] = a.cpu().numpy()
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for k in range(2):
        assert rel_l2(got[k], want[k]) < 1e-6
