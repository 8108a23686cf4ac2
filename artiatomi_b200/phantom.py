"""Seeded synthetic inputs: ellipsoid/bead phantoms and tilt-series alignment.

The benchmark configurations use synthetic phantoms; the reference names no
dataset. A phantom is a sum of ellipsoids with semi-axes U(a_min, a_max)
voxels, densities U(d_min, d_max) and uniformly random orientations, plus
optional gold beads (spheres of radius 5 and density 5.0). The array layout
is [z][y][x], x fastest, as the reconstruction kernels use.
"""
from __future__ import annotations

import math

import numpy as np


def _random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def ellipsoid_list(dims, n_ellipsoids, seed=0, axes=(3.0, 20.0), density=(0.2, 1.0), n_beads=0, bead_radius=5.0,
                   bead_density=5.0):
    """(centre[xyz], inverse-shape matrix, density) tuples, reproducible."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    out = []
    for _ in range(n_ellipsoids):
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        a = rng.uniform(axes[0], axes[1], size=3)
        R = _random_rotation(rng)
        A = R @ np.diag(1.0 / a ** 2) @ R.T
        out.append((c, A, float(rng.uniform(*density)), float(a.max())))
    for _ in range(n_beads):
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        A = np.eye(3) / bead_radius ** 2
        out.append((c, A, float(bead_density), float(bead_radius)))
    return out


def phantom_numpy(dims, n_ellipsoids=200, seed=0, **kw) -> np.ndarray:
    """Rasterise the phantom on the CPU (voxel centres at integer + 0.5)."""
    nx, ny, nz = dims
    vol = np.zeros((nz, ny, nx), np.float32)
    for c, A, d, r in ellipsoid_list(dims, n_ellipsoids, seed, **kw):
        lo = np.maximum(np.floor(c - r - 1).astype(int), 0)
        hi = np.minimum(np.ceil(c + r + 1).astype(int), [nx, ny, nz])
        if np.any(hi <= lo):
            continue
        zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2]) + 0.5, np.arange(lo[1], hi[1]) + 0.5,
                                 np.arange(lo[0], hi[0]) + 0.5, indexing="ij")
        p = np.stack([xx - c[0], yy - c[1], zz - c[2]], -1)
        q = np.einsum("...i,ij,...j->...", p, A, p)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += (q <= 1.0) * np.float32(d)
    return vol


def phantom_torch(dims, n_ellipsoids=200, seed=0, device="cuda", **kw):
    """Same phantom rasterised on the GPU with torch (memory only)."""
    import torch

    nx, ny, nz = dims
    vol = torch.zeros((nz, ny, nx), dtype=torch.float32, device=device)
    for c, A, d, r in ellipsoid_list(dims, n_ellipsoids, seed, **kw):
        lo = np.maximum(np.floor(c - r - 1).astype(int), 0)
        hi = np.minimum(np.ceil(c + r + 1).astype(int), [nx, ny, nz])
        if np.any(hi <= lo):
            continue
        z = torch.arange(lo[2], hi[2], device=device, dtype=torch.float64) + 0.5 - c[2]
        y = torch.arange(lo[1], hi[1], device=device, dtype=torch.float64) + 0.5 - c[1]
        x = torch.arange(lo[0], hi[0], device=device, dtype=torch.float64) + 0.5 - c[0]
        zz, yy, xx = torch.meshgrid(z, y, x, indexing="ij")
        At = torch.tensor(A, device=device)
        q = (At[0, 0] * xx * xx + At[1, 1] * yy * yy + At[2, 2] * zz * zz + 2 * At[0, 1] * xx * yy +
             2 * At[0, 2] * xx * zz + 2 * At[1, 2] * yy * zz)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += (q <= 1.0).to(torch.float32) * d
    return vol


def tilt_series(n_proj, t_min=-60.0, t_max=60.0):
    """Evenly spaced tilt angles in degrees."""
    return np.linspace(t_min, t_max, n_proj).astype(np.float32)


def alignment(n_proj, seed=0, shift=0.0, psi_jitter=0.0):
    """Marker-file items per projection: x/y shifts U(+-shift) px and psi
    U(+-psi_jitter) degrees."""
    rng = np.random.default_rng(seed + 1)
    xs = rng.uniform(-shift, shift, n_proj).astype(np.float32) if shift else np.zeros(n_proj, np.float32)
    ys = rng.uniform(-shift, shift, n_proj).astype(np.float32) if shift else np.zeros(n_proj, np.float32)
    psi = rng.uniform(-psi_jitter, psi_jitter, n_proj).astype(np.float32) if psi_jitter else np.zeros(n_proj, np.float32)
    return xs, ys, psi
