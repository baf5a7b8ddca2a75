"""Random-phase spectral initial condition and energy spectrum (lbm_b200.spectral)."""
import numpy as np
import pytest
import torch

from lbm_b200 import spectral as SP


def test_initial_field_is_divergence_free_and_scaled():
    ux, uy = SP.random_phase_velocity(256, k0=8.0, u_rms=0.05, seed=3)
    assert SP.spectral_divergence(ux, uy) < 1e-12
    assert abs(np.sqrt(np.mean(ux ** 2 + uy ** 2)) - 0.05) < 1e-12
    assert abs(ux.mean()) < 1e-15 and abs(uy.mean()) < 1e-15


def test_spectrum_shape_peak_and_parseval():
    N, k0 = 512, 8.0
    ux, uy = SP.random_phase_velocity(N, k0=k0, u_rms=0.1 * SP.CS, seed=1)
    k, E = SP.energy_spectrum(ux, uy)
    assert abs(E.sum() - 0.5 * np.mean(ux ** 2 + uy ** 2)) < 1e-12 * max(1.0, E.sum()) + 1e-15
    assert abs(int(k[np.argmax(E)]) - k0) <= 2
    sel = (k >= 2) & (k <= 24)
    model = k[sel] ** 4 * np.exp(-2.0 * (k[sel] / k0) ** 2)
    ratio = E[sel] / model
    # shells hold ~2 pi k modes with random phases: scatter of tens of percent
    assert np.corrcoef(np.log(E[sel]), np.log(model))[0, 1] > 0.97
    assert ratio.max() / ratio.min() < 4.0


def test_torch_and_numpy_spectra_agree():
    ux, uy = SP.random_phase_velocity(128, seed=5)
    k1, E1 = SP.energy_spectrum(ux, uy)
    k2, E2 = SP.energy_spectrum(torch.from_numpy(ux), torch.from_numpy(uy))
    assert np.array_equal(k1, k2) and np.allclose(E1, E2, rtol=1e-12, atol=1e-18)


def test_box_filter_and_seeded_state():
    a = np.arange(16.0).reshape(4, 4)
    assert np.array_equal(SP.box_filter(a, 2), np.array([[2.5, 4.5], [10.5, 12.5]]))
    f1 = SP.turbulence_state(64, seed=9)
    f2 = SP.turbulence_state(64, seed=9)
    assert f1.shape == (9, 64, 64) and np.array_equal(f1, f2)
    assert abs(f1.sum(axis=0).mean() - 1.0) < 1e-6


@pytest.mark.gpu
def test_decaying_turbulence_on_gpu():
    """C4-style decay at 256^2 (periodic, MRT + Smagorinsky): the kinetic energy
    falls monotonically and the spectrum from device macros matches the host's."""
    from helpers import dev, host
    from lbm_b200 import solver as SV

    N = 256
    f0 = SP.turbulence_state(N, k0=8.0, u_rms=0.1 * SP.CS, seed=2)
    S = SV.Solver(N, N, bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC, bc_y=SV.BC_PERIODIC, cs_smag=0.1,
                  s_nu=1.0 / (3 * 0.002 + 0.5), ref_clamps=0)
    m = torch.zeros((N, N), dtype=torch.uint8, device="cuda")
    a, b = dev(f0), dev(f0)
    mac = [torch.zeros((N, N), device="cuda") for _ in range(3)]
    energies = []
    for _ in range(5):
        which = S.run(a, b, m, 100, 4, *mac)
        if which:
            a, b = b, a
        energies.append(0.5 * float((mac[0] ** 2 + mac[1] ** 2).mean()))
    assert all(e2 < e1 for e1, e2 in zip(energies, energies[1:]))
    assert energies[-1] > 0.2 * energies[0]
    k, Ed = SP.energy_spectrum(mac[0], mac[1])
    _, Eh = SP.energy_spectrum(host(mac[0]).astype(np.float64), host(mac[1]).astype(np.float64))
    assert np.allclose(Ed, Eh, rtol=1e-9, atol=1e-16)


def test_balanced_density_solves_the_pressure_poisson_equation():
    """rho = 1 + 3 p with lap p = -d_i d_j (u_i u_j) (spectral, periodic)."""
    N = 128  # k0 = 4: the products u_i u_j stay well below the Nyquist wavenumber
    ux, uy = SP.random_phase_velocity(N, 4.0, 0.1 * SP.CS, 5)
    rho = SP.balanced_density(ux, uy)
    p = (rho - 1.0) / 3.0
    k = np.fft.fftfreq(N, d=1.0 / N) * 2.0 * np.pi / N
    ky, kx = np.meshgrid(k, k, indexing="ij")
    F = np.fft.fft2
    lap_p = -(kx * kx + ky * ky) * F(p)
    rhs = (kx * kx * F(ux * ux) + 2.0 * kx * ky * F(ux * uy) + ky * ky * F(uy * uy))
    inner = np.ones((N, N), bool)
    inner[N // 2, :] = inner[:, N // 2] = False  # the Nyquist row and column are not Hermitian for k_x k_y
    assert np.abs((lap_p - rhs)[inner]).max() < 1e-10 * np.abs(rhs).max()  # -k^2 p_hat = k_i k_j (u_i u_j)_hat
    assert abs(p.mean()) < 1e-15
    # vortex cores (high speed) sit at low pressure
    sp = np.hypot(ux, uy)
    assert np.corrcoef(sp.ravel(), p.ravel())[0, 1] < 0
