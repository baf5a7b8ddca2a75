"""Host-side parts of the headless drivers: the drivers' constants, initial
state, MLUPS accounting and PNG writer (no GPU)."""
import numpy as np
import pytest

from lbm_b200 import drivers as D
from lbm_b200 import init as I


def test_driver_constants():
    # lbm_mine2.py:77-79, 90; lbm_smemaa_main.py:95, 107-108, 165;
    # lbm_smemaa_endfused_main.py:61, 67-68, 89
    c = D.DRIVERS
    assert (c["core4"].T, c["core4"].tau_inv, c["core4"].u_in, c["core4"].iters_per_frame) == (1, 1.8, 0.10, 25)
    assert c["core4"].tau_inv_bnd == 1.8
    assert (c["smemaa"].T, c["smemaa"].tau_inv, c["smemaa"].iters_per_frame) == (4, 1.7, 50)
    assert (c["endfused"].T, c["endfused"].tau_inv, c["endfused"].iters_per_frame) == (6, 1.0, 20)
    assert c["endfused"].macro_per_frame and not c["smemaa"].macro_per_frame
    assert D.VORT_SCALE == 50.0


def test_mlups_formula():
    # lbm_mine2.py:106: W * H * iters_per_frame * fps * 2 (two launches of one step)
    assert D.mlups_reference(2048, 512, 25, 2, 100.0) == pytest.approx(2048 * 512 * 25 * 100.0 * 2 / 1e6)
    # lbm_smemaa_main.py:202: W * H * iters_per_frame * (2 T) * fps
    assert D.mlups_reference(2048, 512, 50, 8, 10.0) == pytest.approx(2048 * 512 * 50 * 8 * 10.0 / 1e6)


def test_initial_state_is_the_drivers():
    W, H = 400, 300
    f = D.reference_initial_state(W, H)
    assert f.shape == (9, H, W) and f.dtype == np.float32
    rho = f.astype(np.float64).sum(0)
    ux = (f.astype(np.float64) * I.CX[:, None, None]).sum(0) / rho
    np.testing.assert_allclose(rho, 1.0, atol=2e-6)
    X, Y = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    want = 0.1 * (np.exp(-((X - 150) ** 2 + (Y - 150) ** 2) / 200.0) - np.exp(-((X - 300) ** 2 + (Y - 150) ** 2) / 200.0))
    np.testing.assert_allclose(ux, want, atol=2e-6)


def test_default_mask_is_a_channel_with_a_cylinder():
    m = D.default_mask(256, 64)
    assert set(np.unique(m)) == {0, 1}
    assert m[0].all() and m[-1].all()
    assert not m[1:-1, 0].any() and not m[1:-1, -1].any()
    assert m[32, 64] == 1


def test_png_round_trip(tmp_path):
    img = np.random.default_rng(3).integers(0, 256, (17, 23, 4), dtype=np.uint8)
    p = tmp_path / "x.png"
    D.write_png(str(p), img)
    np.testing.assert_array_equal(D.read_png(str(p)), img)
    raw = p.read_bytes()
    assert raw[:8] == b"\x89PNG\r\n\x1a\n" and raw[12:16] == b"IHDR"


def test_unknown_driver_rejected():
    with pytest.raises(ValueError):
        D.HeadlessDriver("nope")
