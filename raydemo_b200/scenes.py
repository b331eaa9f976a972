"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference ships no benchmark scenes for these configurations, so every
scene here is procedural and fully determined by its seed.
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------- microbench


def random_triangles(n_tris: int, seed: int = 0, mean_edge: float = 0.005, sigma: float = 0.5) -> np.ndarray:
    """`n_tris` random triangles, returned as float32 vertex positions (n, 3, 3).

    Centroids are uniform in the unit cube; each vertex sits at the centroid
    plus an isotropic unit direction times a lognormal(ln mean_edge, sigma)
    length, which gives random orientations and lognormal edge lengths.
    """
    rng = np.random.default_rng(seed)
    c = rng.random((n_tris, 1, 3))
    g = rng.standard_normal((n_tris, 3, 3))
    g /= np.linalg.norm(g, axis=2, keepdims=True)
    length = rng.lognormal(np.log(mean_edge), sigma, (n_tris, 3, 1))
    return (c + g * length).astype(np.float32)


def incoherent_rays(n_rays: int, seed: int = 1, tmax: float = 1e30) -> np.ndarray:
    """Rays as (n, 8) float32: origin uniform in the unit cube, direction
    uniform on the sphere; columns are ox, oy, oz, tmax, dx, dy, dz, 0."""
    rng = np.random.default_rng(seed)
    o = rng.random((n_rays, 3))
    d = rng.standard_normal((n_rays, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n_rays, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    return r


def coherent_rays(w: int = 2048, h: int = 2048, origin=(0.5, 0.5, -1.5), fov_deg: float = 45.0, tmax: float = 1e30) -> np.ndarray:
    """One pinhole ray per pixel centre, looking along +z at the unit cube."""
    o = np.asarray(origin, np.float64)
    k = np.tan(np.radians(fov_deg) * 0.5)
    xs = ((np.arange(w) + 0.5) / w * 2.0 - 1.0) * k * (w / h)
    ys = (1.0 - (np.arange(h) + 0.5) / h * 2.0) * k
    X, Y = np.meshgrid(xs, ys)
    d = np.stack([X, Y, np.ones_like(X)], axis=-1).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((w * h, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    return r


def triangle_soup_mesh(tris: np.ndarray):
    """Vertex attributes (PxyzNxyzTuv, 8 floats per vertex) and indices for a
    triangle soup, as the scene API takes them."""
    n = len(tris)
    attrs = np.zeros((n * 3, 8), np.float32)
    attrs[:, 0:3] = tris.reshape(-1, 3)
    attrs[:, 5] = 1.0
    idx = np.arange(n * 3, dtype=np.uint32)
    return attrs, idx


def tri_aabbs(tris: np.ndarray) -> np.ndarray:
    return np.concatenate([tris.min(axis=1), tris.max(axis=1)], axis=1).astype(np.float32)
