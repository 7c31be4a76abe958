"""Seeded synthetic MRI inputs: trajectories, density weights, images, coil maps.

All generators are written for this library (no reference data is used).
Coordinates are returned in grid units, ``k * N`` with ``k`` in [-0.5, 0.5),
ordered (x, y[, z]) along the last axis — the convention of
``deepmr.fft.plan_nufft`` (src/deepmr/fft/nufft.py:33-36).
"""

import math

import numpy as np
import torch

GOLDEN_ANGLE = math.pi * (math.sqrt(5.0) - 1.0) / 2.0  # radial golden angle (rad)
GOLDEN_MEANS_3D = (0.4656, 0.6823)  # 2D golden means for 3D radial ordering


def radial_2d(nspokes, nsamples, shape, angle_offset=0.0):
    """Golden-angle 2D radial trajectory, (nspokes, nsamples, 2) float32.

    Spoke ``i`` has angle ``i * pi (sqrt5 - 1) / 2``; the readout spans
    ``r = linspace(-0.5, 0.5, nsamples, endpoint=False)``.
    """
    ny, nx = (shape, shape) if np.isscalar(shape) else tuple(shape)[-2:]
    r = np.linspace(-0.5, 0.5, nsamples, endpoint=False)
    phi = angle_offset + np.arange(nspokes) * GOLDEN_ANGLE
    kx = np.cos(phi)[:, None] * r[None, :]
    ky = np.sin(phi)[:, None] * r[None, :]
    return np.stack([kx * nx, ky * ny], axis=-1).astype(np.float32)


def kooshball_3d(nspokes, nsamples, shape):
    """Golden-means 3D radial ("kooshball"), (nspokes, nsamples, 3) float32.

    Spoke ``i`` has polar cosine ``frac(i * 0.4656)`` and azimuth
    ``2 pi frac(i * 0.6823)``; full-diameter readouts ``r`` in [-0.5, 0.5).
    """
    nz, ny, nx = (shape,) * 3 if np.isscalar(shape) else tuple(shape)[-3:]
    i = np.arange(nspokes, dtype=np.float64)
    cz = np.mod(i * GOLDEN_MEANS_3D[0], 1.0)
    az = 2.0 * math.pi * np.mod(i * GOLDEN_MEANS_3D[1], 1.0)
    sz = np.sqrt(1.0 - cz**2)
    d = np.stack([sz * np.cos(az), sz * np.sin(az), cz], axis=-1)  # (x, y, z)
    r = np.linspace(-0.5, 0.5, nsamples, endpoint=False)
    k = d[:, None, :] * r[None, :, None]
    k = k * np.asarray([nx, ny, nz], dtype=np.float64)
    return k.astype(np.float32)


def spiral_2d(nsamples, shape, rotation=0.0, nturns=None, density=1.5):
    """Variable-density single-interleaf spiral, (1, nsamples, 2) float32.

    ``r(t) = 0.5 t**density``, ``phi(t) = 2 pi nturns t + rotation`` for
    ``t = linspace(0, 1, nsamples, endpoint=False)`` (denser at the centre).
    """
    ny, nx = (shape, shape) if np.isscalar(shape) else tuple(shape)[-2:]
    if nturns is None:
        nturns = max(ny, nx) / 8.0
    t = np.linspace(0.0, 1.0, nsamples, endpoint=False)
    r = 0.5 * t**density
    phi = 2.0 * math.pi * nturns * t + rotation
    k = np.stack([r * np.cos(phi) * nx, r * np.sin(phi) * ny], axis=-1)
    k = np.clip(k, -0.5 * np.asarray([nx, ny]), np.nextafter(0.5 * np.asarray([nx, ny]), 0))
    return k[None].astype(np.float32)


def ramp_dcf(coord):
    """Ramp density weights ``|k| / max|k|``; zero-radius samples get 1/nsamples."""
    c = np.asarray(coord, dtype=np.float64)
    r = np.sqrt((c**2).sum(-1))
    rmax = r.max() if r.max() > 0 else 1.0
    w = r / rmax
    w[r == 0] = 1.0 / c.shape[-2]
    return w.astype(np.float32)


def complex_gaussian(shape, seed=0, device="cpu"):
    """i.i.d. standard complex Gaussian (E|x|^2 = 1), complex64."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    re = torch.randn(shape, generator=g, device=device, dtype=torch.float32)
    im = torch.randn(shape, generator=g, device=device, dtype=torch.float32)
    return torch.complex(re, im) * (0.5**0.5)


def ellipse_phantom(shape, seed=0, nellipses=8):
    """Seeded random-ellipse phantom (a Shepp-Logan-like test object), float32.

    Ellipse centres, axes, angles and intensities are drawn from a seeded RNG;
    no published ellipse table is used.
    """
    rng = np.random.default_rng(seed)
    ny, nx = (shape, shape) if np.isscalar(shape) else tuple(shape)[-2:]
    y, x = np.meshgrid(np.linspace(-1, 1, ny), np.linspace(-1, 1, nx), indexing="ij")
    img = np.zeros((ny, nx), dtype=np.float64)
    # outer head shape, then random inner structures
    img[(x / 0.72) ** 2 + (y / 0.92) ** 2 <= 1] = 1.0
    img[(x / 0.66) ** 2 + ((y + 0.02) / 0.86) ** 2 <= 1] -= 0.7
    for _ in range(nellipses):
        cx, cy = rng.uniform(-0.4, 0.4, 2)
        a, b = rng.uniform(0.05, 0.3, 2)
        th = rng.uniform(0, np.pi)
        v = rng.uniform(-0.2, 0.4)
        xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
        yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1] += v
    return img.astype(np.float32)


def coil_maps(ncoils, shape, seed=0):
    """Random-phase Gaussian-magnitude blob coil maps normalised to sum |S|^2 = 1.

    Returns (ncoils, *shape) complex64.
    """
    rng = np.random.default_rng(seed)
    shape = tuple(shape)
    axes = np.meshgrid(*[np.linspace(-1, 1, n) for n in shape], indexing="ij")
    maps = []
    for _ in range(ncoils):
        centre = rng.uniform(-1.2, 1.2, len(shape))
        width = rng.uniform(0.6, 1.4)
        r2 = sum((a - c) ** 2 for a, c in zip(axes, centre))
        mag = np.exp(-r2 / (2 * width**2))
        phase = rng.uniform(-np.pi, np.pi) + sum(
            rng.uniform(-1.5, 1.5) * a for a in axes
        )
        maps.append(mag * np.exp(1j * phase))
    maps = np.stack(maps)
    rss = np.sqrt((np.abs(maps) ** 2).sum(0, keepdims=True))
    return (maps / rss).astype(np.complex64)
