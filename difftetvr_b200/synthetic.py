"""Seeded synthetic inputs: Kuhn-subdivided cube grids with jittered interior
vertices, Gaussian-sum densities and cameras on a sphere.  They stand in for
the reference's datasets (which are neither in this repository nor needed):
same mesh family as TetMesh::setHexMeshConst, same camera construction as
pytests/datasets/sample_view.py:98-130.
"""
from __future__ import annotations

import math

import numpy as np

from .tet_mesh import build_hex_mesh


def kuhn_mesh(n: int, seed: int = 0, jitter: float = 0.2, lo: float = -1.0, hi: float = 1.0):
    """n^3 cubes on [lo, hi]^3 split into 6n^3 tets; interior vertices jittered by
    U(-jitter, jitter) * h per axis (h = cell size).  Returns (cells u32[T,4], positions f32[V,3])."""
    cells, pos = build_hex_mesh((lo, lo, lo), (hi, hi, hi), n + 1, n + 1, n + 1)
    rng = np.random.default_rng(seed)
    h = (hi - lo) / n
    idx = np.arange(pos.shape[0])
    ix = idx % (n + 1)
    iy = (idx // (n + 1)) % (n + 1)
    iz = idx // ((n + 1) * (n + 1))
    interior = (ix > 0) & (ix < n) & (iy > 0) & (iy < n) & (iz > 0) & (iz < n)
    jit = rng.uniform(-jitter, jitter, size=pos.shape) * h
    pos = pos + (jit * interior[:, None]).astype(np.float32)
    return cells, pos.astype(np.float32)


def gaussian_colors(positions: np.ndarray, seed: int = 0, num_gaussians: int = 4):
    """RGB ~ U[0,1]; A = sum of isotropic Gaussians (centres U[-1,1]^3,
    sigma U[0.2,0.5], peak U[1,8])."""
    rng = np.random.default_rng(seed + 7919)
    V = positions.shape[0]
    rgb = rng.uniform(0.0, 1.0, size=(V, 3))
    centres = rng.uniform(-1.0, 1.0, size=(num_gaussians, 3))
    sigma = rng.uniform(0.2, 0.5, size=num_gaussians)
    peak = rng.uniform(1.0, 8.0, size=num_gaussians)
    d2 = ((positions[:, None, :].astype(np.float64) - centres[None]) ** 2).sum(-1)
    a = (peak[None] * np.exp(-d2 / (2.0 * sigma[None] ** 2))).sum(-1)
    return np.concatenate([rgb, a[:, None]], axis=1).astype(np.float32)


def look_at_view(camera_position) -> list[float]:
    """View matrix (column-major 16 floats) of a camera at `camera_position`
    looking at the origin with up = +y (sample_view.py:114-130)."""
    cp = np.asarray(camera_position, dtype=np.float64)
    up = np.array([0.0, 1.0, 0.0])
    fwd = cp / np.linalg.norm(cp)
    right = np.cross(up, fwd)
    right /= np.linalg.norm(right)
    up2 = np.cross(fwd, right)
    up2 /= np.linalg.norm(up2)
    rot = np.eye(4)
    rot[:3, 0], rot[:3, 1], rot[:3, 2] = right, up2, fwd
    trans = np.eye(4)
    trans[:3, 3] = cp
    view = np.linalg.inv(trans @ rot)
    return [float(view[j, i]) for i in range(4) for j in range(4)]


def sphere_camera(seed: int, distance: float = 3.0) -> list[float]:
    """Seeded direction on the unit sphere (|dir . up| <= 0.99), camera at distance."""
    rng = np.random.default_rng(seed + 104729)
    while True:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if abs(d[1]) <= 0.99:
            return look_at_view(d * distance)


def fibonacci_cameras(n: int, distance: float = 3.0) -> list[list[float]]:
    """n cameras on a Fibonacci sphere (poles nudged off the up axis)."""
    out = []
    golden = math.pi * (3.0 - math.sqrt(5.0))
    for i in range(n):
        y = 1.0 - 2.0 * (i + 0.5) / n
        y = max(min(y, 0.98), -0.98)
        r = math.sqrt(1.0 - y * y)
        th = golden * i
        out.append(look_at_view(np.array([r * math.cos(th), y, r * math.sin(th)]) * distance))
    return out


FOVY_45 = math.radians(45.0)
