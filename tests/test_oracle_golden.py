"""Pin the CPU oracle to the reference's own kernels.

tests/golden/*.npz hold outputs of the reference kernels (lbm_core4.cu,
lbm_core_smemaa.cu, lbm_core_smemaa_policy.cu, lbm_core_smemaa_endfused.cu,
compiled from source with -use_fast_math) on seeded inputs, produced on a B200
by tests/golden/make_golden.py.  The oracle (IEEE FP32, no fast math) must
reproduce them within the FP32 parity tolerance (relative L2 1e-5)."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from helpers import REL_TOL, away_from_outlet_corners, rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    path = os.path.join(GOLD, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"missing fixture {name}")
    return np.load(path)


@pytest.mark.parametrize("name", ["core4_64x48", "core4_130x66"])
def test_core4(name):
    d = _load(name)
    W, H = int(d["W"]), int(d["H"])
    a, b = d["f0"].copy(), d["f0"].copy()
    mac = tuple(np.zeros((H, W), np.float32) for _ in range(3))
    for s in range(1, int(d["snaps"].max()) + 1):
        O.core4_step(d["mask"], a, b, mac, tau_inv=float(d["tau_inv"]), u_in=float(d["u_in"]))
        a, b = b, a
        if s in d["snaps"]:
            assert rel_l2(a, d[f"f_{s}"]) < REL_TOL
            for k, m in zip(("ux", "uy", "rho"), mac):
                assert rel_l2(m, d[f"{k}_{s}"]) < REL_TOL, (k, s)


@pytest.mark.parametrize("name", ["smemaa_64x48", "smemaa_130x66"])
def test_smemaa(name):
    d = _load(name)
    W, H, T = int(d["W"]), int(d["H"]), int(d["T"])
    a, b = d["f0"].copy(), d["f0"].copy()
    mac = tuple(np.zeros((H, W), np.float32) for _ in range(3))
    for n in range(1, int(d["snaps"].max()) + 1):
        O.smemaa_launch(d["mask"], a, b, mac, tau_inv=float(d["tau_inv"]), u_in=float(d["u_in"]), T=T)
        a, b = b, a
        if n in d["snaps"]:
            assert rel_l2(a, d[f"f_{n}"]) < REL_TOL
            for k, m in zip(("ux", "uy", "rho"), mac):
                assert rel_l2(m, d[f"{k}_{n}"]) < REL_TOL, (k, n)


@pytest.mark.parametrize("name", ["policy_64x48", "policy_130x66", "endfused_130x66"])
def test_policy_endfused(name):
    """Compared outside the light cone of the outlet corners, where the reference
    reads shared memory it never initialised (helpers.away_from_outlet_corners)."""
    d = _load(name)
    W, H, T = int(d["W"]), int(d["H"]), int(d["T"])
    a, b = d["f0"].copy(), d["f0"].copy()
    for n in range(1, int(d["snaps"].max()) + 1):
        O.policy_launch(d["mask"], a, b, tau_inv=float(d["tau_inv"]), u_in=float(d["u_in"]), T=T)
        a, b = b, a
        if n in d["snaps"]:
            ok = away_from_outlet_corners(W, H, n * T + 2)
            assert rel_l2(a[:, ok], d[f"f_{n}"][:, ok]) < REL_TOL
            mac = O.macro(a, d["mask"], u_in=float(d["u_in"]))
            for k, m in zip(("ux", "uy", "rho"), mac):
                assert rel_l2(m[ok], d[f"{k}_{n}"][ok]) < REL_TOL, (k, n)


def test_visualize():
    d = _load("visualize_96x40")
    img = O.visualize(d["ux"], d["uy"], d["mask"], float(d["vort_scale"]))
    np.testing.assert_array_equal(img, d["img"])


def test_every_fixture_is_checked():
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "*.npz")))
    assert names, "no golden fixtures"
    for n in names:
        assert n.split("_")[0] in ("core4", "smemaa", "policy", "endfused", "visualize"), n
