"""Seeded synthetic inputs in place of the reference's MATLAB data generator.

The reference samples points on .wrl meshes (matlab/new_data.m:180-200) and
draws den = randn + i*rand (new_data.m:201).  The workloads here are analytic
surfaces instead:
  * sphere of diameter K centred in the root box of width K, points uniform
    by area;
  * ellipsoid with semi-axes (0.5, 0.25, 0.125) * K, uniform by area
    (rejection on the area element);
densities complex with real and imaginary parts i.i.d. N(0,1).  Coordinates
are in wavelengths (the kernel wavenumber is 2*pi, src/kernel3d.cpp:33).
Points are scaled by (1 - 1e-12) so the surface never touches the root-box
faces, where setup_tree's cell index check would fail
(src/wave3d_setup.cpp:124-128).
"""
from __future__ import annotations

import math

import numpy as np

SHRINK = 1.0 - 1e-12


def sphere_points(n: int, K: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * (0.5 * K * SHRINK)


def ellipsoid_points(n: int, K: float, seed: int = 0, axes=(0.5, 0.25, 0.125)) -> np.ndarray:
    """Uniform-by-area samples: draw on the unit sphere, map to the
    ellipsoid, accept with probability proportional to the area element
    |J| = abc * |x/a^2, y/b^2, z/c^2| (relative to its maximum)."""
    rng = np.random.default_rng(seed)
    a, b, c = (s * K * SHRINK for s in axes)
    out = []
    have = 0
    gmax = a * b * c / min(a, b, c)
    while have < n:
        u = rng.standard_normal((2 * n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        p = u * np.array([a, b, c])
        g = a * b * c * np.sqrt((p[:, 0] / a ** 2) ** 2 + (p[:, 1] / b ** 2) ** 2 + (p[:, 2] / c ** 2) ** 2)
        keep = rng.random(2 * n) * gmax < g
        out.append(p[keep])
        have += int(keep.sum())
    return np.concatenate(out)[:n]


def cluster_points(n: int, K: float, seed: int = 0) -> np.ndarray:
    """Strongly non-uniform cloud for adaptive trees: half the points on a
    sphere of diameter 0.8 K, the rest in three tight Gaussian blobs, plus a
    few exact duplicates (coincident pairs exercise the r := 1 rule of
    src/kernel3d.cpp:47-49)."""
    rng = np.random.default_rng(seed)
    n_s = n // 2
    v = rng.standard_normal((n_s, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    parts = [v * 0.4 * K]
    centres = np.array([[0.2, 0.1, -0.15], [-0.25, 0.2, 0.1], [0.05, -0.3, 0.3]]) * K
    n_b = n - n_s - 8
    for i in range(3):
        m = n_b // 3 + (1 if i < n_b % 3 else 0)
        parts.append(centres[i] + rng.standard_normal((m, 3)) * (0.02 * K))
    pts = np.concatenate(parts)
    pts = np.clip(pts, -0.5 * K * SHRINK, 0.5 * K * SHRINK)
    dup = pts[rng.choice(pts.shape[0], size=8, replace=False)]
    return np.concatenate([pts, dup])


def sphere_n_for(K: float, pts_per_wl2: float = 25.0) -> int:
    """N for a sphere of diameter K at a given density (area pi K^2)."""
    return int(round(pts_per_wl2 * math.pi * K * K))


def densities(n: int, seed: int = 0, dtype=np.complex128) -> np.ndarray:
    rng = np.random.default_rng(seed)
    re = rng.standard_normal(n)
    im = rng.standard_normal(n)
    return (re + 1j * im).astype(dtype)


def check_ids(n: int, count: int = 200, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed + 7919)
    count = min(count, n)
    return np.sort(rng.choice(n, size=count, replace=False)).astype(np.int32)


def cells_for(K: float) -> int:
    """Cell-level partition size NC = min(8, K), the reference's practice at
    K=64 (matlab/data_script.m:31-35); must be a power of two with K/NC >= 1."""
    nc = 1
    while nc * 2 <= min(8, K):
        nc *= 2
    return nc


def maxlevel_for(K: float) -> int:
    return int(round(math.log2(K))) + 6
