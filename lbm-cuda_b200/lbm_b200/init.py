"""Initial-state and mask builders (host side, numpy).

These reproduce the reference drivers' conventions:

* equilibrium initial state from (rho, u_x, u_y) with the second-order BGK
  equilibrium, lbm_mine2.py:28-36;
* the Gaussian-pair initial velocity of the drivers, lbm_mine2.py:19-26;
* mask conventions, lbm_mine2.py:39-58: True = solid, rows 0 and H-1 solid,
  columns 0 and W-1 forced fluid on the interior rows.  The reference loads its
  obstacle from ``circle.bmp`` (green channel == 0 -> solid); that image is not
  part of the reference tree, so procedural cylinders and discs are provided
  next to an image loader with the same rule.

Arrays are C-ordered: masks ``(H, W)`` uint8, populations ``(9, H, W)`` float32
(plane q is ``f[q]``), which is the SoA layout ``f[q*W*H + y*W + x]`` of the
reference kernels.
"""
from __future__ import annotations

import numpy as np

CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.int64)
CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.int64)
OPP = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6], dtype=np.int64)
WEIGHTS = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=np.float64)

# Mask byte values understood by the general solver (lbm_params).  The reference
# kernels treat any nonzero byte as solid, so a mask built with FLUID/SOLID only
# is also a valid reference mask.
FLUID = 0
SOLID = 1
MOVING_WALL = 2  # Ladd moving-wall bounce-back with the lid velocity
OBSTACLE = 3  # solid, and counted by the drag/lift momentum exchange


def equilibrium(rho, ux, uy, dtype=np.float32) -> np.ndarray:
    """f_q = w_q rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2), lbm_mine2.py:30-34."""
    rho = np.asarray(rho, dtype=np.float64)
    ux = np.asarray(ux, dtype=np.float64)
    uy = np.asarray(uy, dtype=np.float64)
    shape = np.broadcast(rho, ux, uy).shape
    f = np.empty((9,) + shape, dtype=np.float64)
    usq = ux * ux + uy * uy
    for q in range(9):
        eu = CX[q] * ux + CY[q] * uy
        f[q] = WEIGHTS[q] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq)
    return f.astype(dtype)


def gaussian_pair_ux(W: int, H: int, amp: float = 0.1, sigma: float = 10.0,
                     c1=(150.0, 150.0), c2=(300.0, 150.0)) -> np.ndarray:
    """u_x = amp (G(c1) - G(c2)), the drivers' initial velocity (lbm_mine2.py:23-26)."""
    X, Y = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    t1 = np.exp(-((X - c1[0]) ** 2 + (Y - c1[1]) ** 2) / (2 * sigma ** 2))
    t2 = np.exp(-((X - c2[0]) ** 2 + (Y - c2[1]) ** 2) / (2 * sigma ** 2))
    return amp * (t1 - t2)


def channel_mask(W: int, H: int) -> np.ndarray:
    """Rows 0 and H-1 solid, columns 0 and W-1 fluid on interior rows (lbm_mine2.py:49-53)."""
    m = np.zeros((H, W), dtype=np.uint8)
    m[0, :] = SOLID
    m[H - 1, :] = SOLID
    return m


def _finish_channel(m: np.ndarray) -> np.ndarray:
    H, W = m.shape
    m[0, :] = SOLID
    m[H - 1, :] = SOLID
    m[1:H - 1, 0] = FLUID
    m[1:H - 1, W - 1] = FLUID
    return m


def add_disc(m: np.ndarray, cx: float, cy: float, radius: float, value: int = OBSTACLE) -> np.ndarray:
    H, W = m.shape
    X, Y = np.meshgrid(np.arange(W), np.arange(H))
    m[(X - cx) ** 2 + (Y - cy) ** 2 <= radius ** 2] = value
    return m


def cylinder_mask(W: int, H: int, cx: float, cy: float, diameter: float, value: int = OBSTACLE) -> np.ndarray:
    """Channel with one circular obstacle; the inlet/outlet columns stay fluid."""
    m = channel_mask(W, H)
    add_disc(m, cx, cy, diameter / 2.0, value)
    return _finish_channel(m)


def random_discs_mask(W: int, H: int, n: int, rmin: float, rmax: float, seed: int,
                      value: int = OBSTACLE) -> np.ndarray:
    """Channel with ``n`` random discs (radius in [rmin, rmax]) away from the open ends."""
    rng = np.random.default_rng(seed)
    m = channel_mask(W, H)
    for _ in range(n):
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(min(W - 1, r + 4), max(r + 4, W - r - 4))
        cy = rng.uniform(min(H - 1, r + 2), max(r + 2, H - r - 2))
        add_disc(m, cx, cy, r, value)
    return _finish_channel(m)


def cavity_mask(W: int, H: int) -> np.ndarray:
    """Lid-driven cavity: solid frame, top row a moving wall (Ladd)."""
    m = np.zeros((H, W), dtype=np.uint8)
    m[0, :] = SOLID
    m[:, 0] = SOLID
    m[:, W - 1] = SOLID
    m[H - 1, :] = MOVING_WALL
    return m


def mask_from_image(path: str, W: int, H: int) -> np.ndarray:
    """Image mask with the reference's rule: green channel == 0 -> solid (lbm_mine2.py:39-58)."""
    import cv2  # optional dependency, only needed for image masks

    img = cv2.imread(path)
    if img is None:
        raise FileNotFoundError(path)
    img = cv2.resize(img, (W, H))
    m = (img[:, :, 1] == 0).astype(np.uint8)
    return _finish_channel(m)


def channel_state(W: int, H: int, u0: float = 0.0, noise: float = 0.0, seed: int = 0,
                  dtype=np.float32) -> np.ndarray:
    """Equilibrium at rho = 1, u = (u0, noise * U(-1, 1)) seeded (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    uy = noise * rng.uniform(-1.0, 1.0, size=(H, W)) if noise else np.zeros((H, W))
    return equilibrium(np.ones((H, W)), np.full((H, W), u0), uy, dtype=dtype)


def perturbed_state(W: int, H: int, seed: int, amp: float = 0.02, dtype=np.float32) -> np.ndarray:
    """Equilibrium of a seeded smooth random velocity and density field (test inputs)."""
    rng = np.random.default_rng(seed)
    X, Y = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    ux = np.zeros((H, W))
    uy = np.zeros((H, W))
    rho = np.ones((H, W))
    for _ in range(4):
        kx, ky = rng.uniform(0.02, 0.2, size=2)
        px, py = rng.uniform(0, 2 * np.pi, size=2)
        ux += amp * np.sin(kx * X + px) * np.cos(ky * Y + py)
        uy += amp * np.cos(kx * X + py) * np.sin(ky * Y + px)
        rho += 0.25 * amp * np.sin(kx * X + ky * Y + px)
    ux += 0.05
    return equilibrium(rho, ux, uy, dtype=dtype)
