"""Lid-driven cavity, the reference configuration's first case: 256 x 256,
plain MRT (s_e 1.1, s_eps 1.0, s_q 1.2, s_nu = 1 / (3 nu + 1/2)), Re = 1000
(nu = 0.0256), lid u = 0.1 through Ladd's moving-wall bounce-back.  The
configuration's 10 000 steps are about four lid passes, while the vortex is
still forming (return flow only -0.09 U, in the upper half); at 60 000 steps
the flow is close to steady and the test checks the known centre-line
structure of the Re = 1000 primary vortex (clockwise for a lid moving in +x):
the return-flow minimum of u on the vertical centre line near -0.37 U low in
the cavity, the v extremes on the horizontal centre line near +0.35 U close to
the left wall and -0.5 U close to the right wall, the layer dragged by the lid,
and mass conservation."""
import numpy as np
import pytest
import torch

from helpers import dev, host
from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu


def test_cavity_re1000_centreline_structure():
    N, U, nu, n = 256, 0.1, 0.0256, 60000
    m = I.cavity_mask(N, N)
    S = SV.Solver(N, N, collision=SV.COLL_MRT, closure=SV.CLOSURE_NONE, bc_left=SV.BC_WALL, bc_right=SV.BC_WALL,
                  bc_y=SV.BC_WALL, s_e=1.1, s_eps=1.0, s_q=1.2, s_nu=1.0 / (3 * nu + 0.5), u_lid=U, ref_clamps=0)
    f0 = I.equilibrium(np.ones((N, N)), np.zeros((N, N)), np.zeros((N, N)))
    a, b = dev(f0), dev(f0)
    md = dev(m)
    d0 = S.diag(a, md).cpu().numpy()
    mac = [torch.zeros((N, N), device="cuda") for _ in range(3)]
    which = S.run(a, b, md, n, 2, *mac)
    f = b if which else a
    d1 = S.diag(f, md).cpu().numpy()
    ux, uy = host(mac[0]) / U, host(mac[1]) / U
    assert np.isfinite(ux).all() and np.isfinite(uy).all()
    assert abs(d1[0] - d0[0]) < 1e-6 * d0[0]
    c = N // 2
    col = ux[1:N - 1, c]          # u on the vertical centre line, y upwards
    row = uy[c, 1:N - 1]          # v on the horizontal centre line
    ymin = np.argmin(col) / (N - 2)
    assert -0.42 < col.min() < -0.32 and 0.12 < ymin < 0.25     # return flow low in the cavity
    assert col[-3:].mean() > 0.8                                 # dragged along under the lid
    xmax, xmin = np.argmax(row) / (N - 2), np.argmin(row) / (N - 2)
    assert 0.30 < row.max() < 0.42 and 0.10 < xmax < 0.25        # upward near the left wall
    assert -0.56 < row.min() < -0.45 and 0.85 < xmin < 0.95      # downward near the right wall
