"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference publishes no input decks for these cases (its placement files
are not part of the tree), so every workload here is generated from a seed:

  vertical_lattice   straight vertical filaments on a square lattice above the
                     wall (the plain-matvec configuration: 4x4 x 20 segments,
                     spacing 20, base height 2, segment spacing 2.2)
  lattice_bases      filament base positions of the reference's rectangular
                     wall seeding (swimmer.cpp:185-257)
  fibonacci_sphere   quasi-uniform points on a sphere (body blobs)
"""
from __future__ import annotations

import numpy as np


def vertical_lattice(nx: int = 4, ny: int = 4, nseg: int = 20, spacing: float = 20.0, base_z: float = 2.0,
                     seg_sep: float = 2.2) -> np.ndarray:
    """Segment centres [nx*ny*nseg, 3] of straight vertical filaments, filament-major order."""
    xs = []
    for i in range(nx):
        for j in range(ny):
            x0 = (i - 0.5 * (nx - 1)) * spacing
            y0 = (j - 0.5 * (ny - 1)) * spacing
            for k in range(nseg):
                xs.append((x0, y0, base_z + seg_sep * k))
    return np.asarray(xs, dtype=np.float64)


def lattice_bases(n_fil: int, fil_x_dim: int, spacing: float, base_height: float) -> np.ndarray:
    """Rectangular wall lattice of the reference (swimmer.cpp:113-185, RECTANGULAR_SEEDING):
    dim_x = min(NFIL, FIL_X_DIM), dim_y = ceil(NFIL/dim_x), fil_id = j + i*dim_y."""
    dim_x = min(n_fil, int(fil_x_dim))
    dim_y = max(1, int(np.ceil(n_fil / dim_x)))
    im = 0.5 * (dim_x - 1.0)
    jm = 0.5 * (dim_y - 1.0)
    out = np.zeros((n_fil, 3))
    for i in range(dim_x):
        for j in range(dim_y):
            fid = j + i * dim_y
            if fid < n_fil:
                out[fid] = ((i - im) * spacing, (j - jm) * spacing, base_height)
    return out


def fibonacci_sphere(n: int, radius: float, centre=(0.0, 0.0, 0.0)) -> np.ndarray:
    """n quasi-uniform points on a sphere (golden-angle spiral)."""
    k = np.arange(n) + 0.5
    z = 1.0 - 2.0 * k / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = np.pi * (3.0 - np.sqrt(5.0)) * k
    pts = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1) * radius
    return pts + np.asarray(centre)


def random_forces(n: int, dof: int, seed: int) -> np.ndarray:
    """Forces (and torques) i.i.d. N(0,1), [n, dof]."""
    return np.random.default_rng(seed).standard_normal((n, dof))


def sphere_with_cilia(n_cilia: int = 1000, nseg: int = 20, n_body: int = 10000, radius: float = 100.0,
                      seg_sep: float = 2.2, centre=(512.0, 512.0, 512.0)):
    """Spherical body of `radius` with `n_body` blobs on a Fibonacci sphere and `n_cilia`
    straight radial cilia of `nseg` segments (first segment seg_sep outside the surface).
    Returns (segment centres [n_cilia*nseg, 3], blob centres [n_body, 3])."""
    c = np.asarray(centre, float)
    blobs = fibonacci_sphere(n_body, radius, c)
    dirs = fibonacci_sphere(n_cilia, 1.0)
    k = np.arange(1, nseg + 1)[None, :, None]
    segs = c + dirs[:, None, :] * (radius + seg_sep * k)
    return segs.reshape(-1, 3), blobs
