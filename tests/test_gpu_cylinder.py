"""Vortex shedding behind a cylinder (the channel configuration at a quarter of
its size): Zou-He inlet u = 0.05 with the reference's wall taper, outflow,
walls, MRT + Smagorinsky (Cs = 0.1), D = 32 in a 1024 x 256 channel, Re = 1000.
Drag and lift come from lbm_forces_fp64 every 50 steps; over the second half of
60 000 steps the lift oscillates at the Strouhal number of a shedding cylinder
(about 0.2; accepted 0.15 .. 0.30) and the mean drag coefficient is of order
one (accepted 0.8 .. 3.0, the blockage D/H = 1/8 raises it)."""
import numpy as np
import pytest
import torch

from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu


def test_cylinder_sheds_vortices_at_strouhal_0_2():
    W, H, D, u = 1024, 256, 32.0, 0.05
    nu = u * D / 1000.0
    mask = torch.from_numpy(I.cylinder_mask(W, H, 256, 128, D, value=I.OBSTACLE)).cuda()
    f = torch.from_numpy(I.channel_state(W, H, u0=0.0, noise=1e-4, seed=0)).cuda()
    g = f.clone()
    S = SV.Solver(W, H, cs_smag=0.1, u_in=u, s_nu=1.0 / (3.0 * nu + 0.5))
    every, n = 50, 1200
    F = torch.zeros((n, 2), dtype=torch.float64, device="cuda")
    for i in range(n):
        if S.run(f, g, mask, every, 2):
            f, g = g, f
        S.forces(f, mask, out=F[i])
    F = F.cpu().numpy()
    assert np.isfinite(F).all()
    q = 0.5 * u * u * D
    cd, cl = F[n // 2:, 0] / q, F[n // 2:, 1] / q
    x = cl - cl.mean()
    spec = np.abs(np.fft.rfft(x * np.hanning(x.size))) ** 2
    freq = np.fft.rfftfreq(x.size, d=float(every))
    st = freq[1 + int(np.argmax(spec[1:]))] * D / u
    assert 0.15 < st < 0.30, st
    assert 0.8 < cd.mean() < 3.0, cd.mean()
    assert np.sqrt(np.mean(x ** 2)) > 0.05  # the lift really oscillates
