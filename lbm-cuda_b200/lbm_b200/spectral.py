"""Decaying-turbulence tools: the random-phase spectral initial condition and the
shell-averaged kinetic energy spectrum (periodic square domains).

Initial condition (the decaying 2-D turbulence configuration): a velocity field
whose energy spectrum is E(k) ~ k^4 exp(-2 (k / k0)^2), with independent uniform
random phases per Fourier mode, projected onto divergence-free fields
(u_hat <- u_hat - k (k . u_hat) / |k|^2) and scaled to a prescribed RMS speed
(u_rms = 0.1 c_s for Mach ~ 0.1 at c_s = 1/sqrt(3)).  The populations start at
the equilibrium of rho = 1 and that velocity.

Spectrum: E(k) = sum over modes with k - 1/2 <= |k| < k + 1/2 of
|u_hat|^2 + |v_hat|^2, divided by 2 N^4 (numpy's unnormalised FFT), so that
sum_k E(k) equals the mean kinetic energy 0.5 <u^2 + v^2> (Parseval).  The FFT is
numpy's on the host or torch's (cuFFT) for device tensors.
"""
from __future__ import annotations

import numpy as np

CS = 1.0 / np.sqrt(3.0)


def _wavenumbers(N: int):
    k = np.fft.fftfreq(N, d=1.0 / N)
    ky, kx = np.meshgrid(k, k, indexing="ij")
    return kx, ky


def random_phase_velocity(N: int, k0: float = 8.0, u_rms: float = 0.1 * CS, seed: int = 0):
    """(ux, uy) float64 arrays (N, N): divergence-free, E(k) ~ k^4 exp(-2 (k/k0)^2)."""
    rng = np.random.default_rng(seed)
    kx, ky = _wavenumbers(N)
    kk = np.hypot(kx, ky)
    amp = np.zeros_like(kk)
    nz = kk > 0
    # E(k) dk spread over the shell circumference 2 pi k: |u_hat(k)|^2 ~ E(k) / k
    amp[nz] = np.sqrt(kk[nz] ** 4 * np.exp(-2.0 * (kk[nz] / k0) ** 2) / kk[nz])
    ph1 = np.exp(2j * np.pi * rng.random((N, N)))
    ph2 = np.exp(2j * np.pi * rng.random((N, N)))
    uh = amp * ph1
    vh = amp * ph2
    # incompressible projection
    k2 = np.where(nz, kk ** 2, 1.0)
    div = (kx * uh + ky * vh) / k2
    uh = uh - kx * div
    vh = vh - ky * div
    ux = np.real(np.fft.ifft2(uh))
    uy = np.real(np.fft.ifft2(vh))
    # the real part of a field with random phases is itself divergence-free
    # (the projection commutes with taking the Hermitian part); remove the mean
    ux -= ux.mean()
    uy -= uy.mean()
    s = u_rms / np.sqrt(np.mean(ux ** 2 + uy ** 2))
    return ux * s, uy * s


def balanced_density(ux, uy, rho0: float = 1.0):
    """Density whose pressure balances an incompressible periodic velocity field:
    the pressure Poisson equation lap p = -d_i d_j (u_i u_j), solved spectrally
    (p_hat = -k_i k_j (u_i u_j)_hat / |k|^2, zero mean), and rho = rho0 (1 + p / c_s^2)
    with c_s^2 = 1/3.  Starting a decaying-turbulence run from this density
    instead of a uniform one removes the acoustic pulse of the vortex cores'
    missing pressure dip, which on large grids steepens into grid-scale waves."""
    ux = np.asarray(ux, dtype=np.float64)
    uy = np.asarray(uy, dtype=np.float64)
    N = ux.shape[0]
    kx, ky = _wavenumbers(N)
    kx = kx * (2.0 * np.pi / N)
    ky = ky * (2.0 * np.pi / N)
    k2 = kx * kx + ky * ky
    k2[0, 0] = 1.0
    rhs = (kx * kx * np.fft.fft2(ux * ux) + 2.0 * kx * ky * np.fft.fft2(ux * uy) + ky * ky * np.fft.fft2(uy * uy))
    ph = -rhs / k2
    ph[0, 0] = 0.0
    p = np.real(np.fft.ifft2(ph))
    return rho0 * (1.0 + 3.0 * p)


def spectral_divergence(ux, uy) -> float:
    """max |k . u_hat| / max |k| |u_hat| (0 for a divergence-free periodic field)."""
    N = ux.shape[0]
    kx, ky = _wavenumbers(N)
    uh, vh = np.fft.fft2(ux), np.fft.fft2(uy)
    d = np.abs(kx * uh + ky * vh).max()
    n = (np.hypot(kx, ky) * np.hypot(np.abs(uh), np.abs(vh))).max()
    return float(d / n)


def energy_spectrum(ux, uy):
    """(k, E) with k = 0 .. N/2 (integers) for square periodic fields (numpy or torch)."""
    try:
        import torch

        if isinstance(ux, torch.Tensor):
            N = ux.shape[0]
            uh = torch.fft.fft2(ux.double())
            vh = torch.fft.fft2(uy.double())
            e = (uh.abs() ** 2 + vh.abs() ** 2) / (2.0 * N ** 4)
            k = torch.fft.fftfreq(N, d=1.0 / N, device=ux.device, dtype=torch.float64)
            kk = torch.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
            idx = torch.round(kk).long().clamp(max=N // 2 + 1)
            E = torch.zeros(N // 2 + 2, dtype=torch.float64, device=ux.device).index_add_(0, idx.flatten(),
                                                                                        e.flatten())
            return np.arange(N // 2 + 1), E[:N // 2 + 1].cpu().numpy()
    except ImportError:
        pass
    ux = np.asarray(ux, dtype=np.float64)
    uy = np.asarray(uy, dtype=np.float64)
    N = ux.shape[0]
    uh, vh = np.fft.fft2(ux), np.fft.fft2(uy)
    e = (np.abs(uh) ** 2 + np.abs(vh) ** 2) / (2.0 * N ** 4)
    kx, ky = _wavenumbers(N)
    idx = np.minimum(np.rint(np.hypot(kx, ky)).astype(int), N // 2 + 1)
    E = np.bincount(idx.ravel(), weights=e.ravel(), minlength=N // 2 + 2)
    return np.arange(N // 2 + 1), E[:N // 2 + 1]


def box_filter(a, f: int):
    """Mean over f x f blocks (the coarse-graining of the high-resolution judge)."""
    a = np.asarray(a)
    N0, N1 = a.shape[-2], a.shape[-1]
    return a.reshape(a.shape[:-2] + (N0 // f, f, N1 // f, f)).mean(axis=(-3, -1))


def turbulence_state(N: int, k0: float = 8.0, u_rms: float = 0.1 * CS, seed: int = 0, dtype=np.float32,
                     balanced: bool = False):
    """Equilibrium populations (9, N, N) of the random-phase velocity and rho = 1
    (or, balanced, the density of :func:`balanced_density`)."""
    from .init import equilibrium

    ux, uy = random_phase_velocity(N, k0, u_rms, seed)
    rho = balanced_density(ux, uy) if balanced else np.ones((N, N))
    return equilibrium(rho, ux, uy, dtype=dtype)
