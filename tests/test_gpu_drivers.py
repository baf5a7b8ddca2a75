"""Headless reference drivers (lbm_b200.drivers) on the GPU.

Each driver captures the reference drivers' CUDA graph of two launches
(f_now -> f_out -> f_now) and replays it `iters_per_frame` times per frame,
then (end-fused driver) the macro kernel and the colour map.  Checks: the
graph-replayed frames give exactly the state and image of the same launches
issued eagerly; the frames agree with the oracle's emulation of the driver loop
(relative L2 <= 1e-5 on the populations and u, v, rho; the image exact on the
GPU's u, v and within one level of the oracle's); the split launch (edge tiles on a forked stream, register wavefront
inside) is captured into the graph correctly; MLUPS follows the drivers'
formula; PNG output round-trips."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, rel_l2
from lbm_b200 import drivers as D

pytestmark = pytest.mark.gpu


def _oracle_frames(kind, mask, f0, frames, iters):
    """The driver loop on the CPU oracle: (f_now, (ux, uy, rho), image)."""
    c = D.DRIVERS[kind]
    H, W = mask.shape
    a, b = f0.copy(), f0.copy()
    mac = (np.zeros((H, W), np.float32), np.zeros((H, W), np.float32), np.ones((H, W), np.float32))
    img = None
    for _ in range(frames):
        for _ in range(iters):
            for src, dst in ((a, b), (b, a)):
                if kind == "core4":
                    O.core4_step(mask, src, dst, mac, tau_inv=c.tau_inv, u_in=c.u_in)
                elif kind == "smemaa":
                    O.smemaa_launch(mask, src, dst, mac, tau_inv=c.tau_inv, u_in=c.u_in, T=c.T)
                else:
                    O.policy_launch(mask, src, dst, tau_inv=c.tau_inv, u_in=c.u_in, T=c.T)
        if c.macro_per_frame:
            O.macro(a, mask, mac, u_in=c.u_in)
        img = O.visualize(mac[0], mac[1], mask, D.VORT_SCALE)
    return a, mac, img


def _host(d):
    torch.cuda.synchronize()
    return (d.f_now.cpu().numpy(), tuple(t.cpu().numpy() for t in (d.ux, d.uy, d.rho)), d.image.cpu().numpy())


@pytest.mark.parametrize("kind", ["core4", "smemaa", "endfused"])
@pytest.mark.parametrize("W,H", [(130, 66), (256, 96)])
def test_driver_graph_vs_eager_and_oracle(kind, W, H):
    mask = D.default_mask(W, H)
    f0 = D.reference_initial_state(W, H)
    frames, iters = 2, 3
    outs = []
    for use_graph in (True, False):
        d = D.HeadlessDriver(kind, W, H, mask=mask, f0=f0, iters_per_frame=iters, use_graph=use_graph)
        for _ in range(frames):
            d.frame()
        outs.append(_host(d))
    (fg, mg, ig), (fe, me, ie) = outs
    np.testing.assert_array_equal(fg, fe)
    for x, y in zip(mg, me):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(ig, ie)
    fo, mo, io = _oracle_frames(kind, mask, f0, frames, iters)
    assert rel_l2(fg, fo) < REL_TOL
    for x, y in zip(mg, mo):
        assert rel_l2(x, y) < REL_TOL
    # the colour map is exact on the GPU's own u, v; against the oracle's frame a
    # byte may differ by one level (near-zero vorticity sits on a truncation edge)
    np.testing.assert_array_equal(ig, O.visualize(mg[0], mg[1], mask, D.VORT_SCALE))
    assert np.abs(ig.astype(np.int16) - io.astype(np.int16)).max() <= 1


@pytest.mark.parametrize("kind", ["smemaa", "endfused"])
def test_driver_graph_captures_split_launch(kind):
    """At 2048 x 2048 (>= 4 M cells, TMA-aligned) each launch is the split form
    with a forked side stream; captured, it must replay to the eager result."""
    W = H = 2048
    mask = D.default_mask(W, H)
    f0 = D.reference_initial_state(W, H)
    res = []
    for use_graph in (True, False):
        d = D.HeadlessDriver(kind, W, H, mask=mask, f0=f0, iters_per_frame=2, use_graph=use_graph)
        d.frame()
        res.append(_host(d))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][2], res[1][2])


@pytest.mark.parametrize("kind", ["core4", "smemaa", "endfused"])
def test_driver_default_size_run_and_png(kind, tmp_path):
    """The drivers' own 2048 x 512 domain and frame constants: run, MLUPS by the
    drivers' formula, a finite state, and the frame written as a PNG."""
    d = D.HeadlessDriver(kind)
    r = d.run(3)
    c = D.DRIVERS[kind]
    assert r["physical_steps"] == 3 * c.iters_per_frame * 2 * c.T
    assert r["mlups"] == pytest.approx(2048 * 512 * c.iters_per_frame * 2 * c.T * r["fps"] / 1e6)
    assert r["mlups_device"] >= r["mlups"] * 0.99  # the host clock includes launch and sync overhead
    assert torch.isfinite(d.f_now).all()
    p = tmp_path / "frame.png"
    d.save_png(str(p))
    np.testing.assert_array_equal(D.read_png(str(p)), d.image_host())


def test_driver_command_line(tmp_path):
    """python -m lbm_b200.drivers: prints the drivers' FPS / MLUPS line and a JSON
    summary, and writes the last frame as a PNG."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=os.path.join(root, "lbm-cuda_b200"))
    png = tmp_path / "frame.png"
    out = subprocess.run([sys.executable, "-m", "lbm_b200.drivers", "--kind", "smemaa", "--W", "512", "--H", "128",
                          "--frames", "12", "--iters-per-frame", "5", "--png", str(png)],
                         env=env, capture_output=True, text=True, timeout=300, check=True).stdout
    assert "[LBM Simulation] FPS:" in out and "MLUPS:" in out
    res = json.loads(out.strip().splitlines()[-1])
    assert res["frames"] == 12 and res["physical_steps"] == 12 * 5 * 8 and res["mlups"] > 0
    img = D.read_png(str(png))
    assert img.shape == (128, 512, 4) and (img[1:-1, 1:-1, 3] == 255).all()
