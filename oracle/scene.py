"""Synthetic inputs of the benchmark workloads, restated for the oracle side.

TEST INFRASTRUCTURE ONLY: the timed CPU implementation (bench.py --impl
reference) builds its inputs here so that it loads no code of the product
library.  Everything is plain numpy and must give the same arrays bit for bit
as difftetvr_b200.synthetic (tests/test_oracle_scene.py checks that):

- kuhn_grid: TetMesh::setHexMeshConst (src/Tet/TetMesh.cpp:1882-1936) with
  HEX_TO_TET_TABLE (:104-117): vertex (ix, iy, iz) at index
  iz * xs * ys + iy * xs + ix, positions lo + (i / (n - 1)) * (hi - lo) in
  FP32, six tets per cube around the diagonal 0-6;
- kuhn_mesh: interior vertices jittered by U(-jitter, jitter) * h per axis;
- gaussian_colors: RGB ~ U[0, 1], density = sum of isotropic Gaussians;
- sphere_camera / look_at_view: camera at distance 3 on a seeded direction,
  looking at the origin (pytests/datasets/sample_view.py:114-130).
"""
from __future__ import annotations

import math

import numpy as np

HEX_TO_TET = np.array([[0, 4, 7, 6], [0, 4, 6, 5], [0, 3, 6, 7], [0, 3, 2, 6], [0, 1, 5, 6], [0, 1, 6, 2]],
                      np.int64)
FOVY_45 = math.radians(45.0)


def kuhn_grid(lo, hi, xs: int, ys: int, zs: int):
    """(cells u32[T, 4], positions f32[V, 3]) of an xs x ys x zs vertex grid."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    iz, iy, ix = np.meshgrid(np.arange(zs), np.arange(ys), np.arange(xs), indexing="ij")
    pos = np.empty((xs * ys * zs, 3), np.float32)
    for k, (i, n) in enumerate(((ix, xs), (iy, ys), (iz, zs))):
        frac = i.reshape(-1).astype(np.float32) / np.float32(n - 1)
        pos[:, k] = lo[k] + frac * (hi[k] - lo[k])
    dy, dz = xs, xs * ys
    cz, cy, cx = np.meshgrid(np.arange(zs - 1), np.arange(ys - 1), np.arange(xs - 1), indexing="ij")
    b = (cz * dz + cy * dy + cx).reshape(-1).astype(np.int64)
    hexv = np.stack([b, b + 1, b + 1 + dy, b + dy, b + dz, b + 1 + dz, b + 1 + dy + dz, b + dy + dz], 1)
    cells = hexv[:, HEX_TO_TET].reshape(-1, 4)
    return cells.astype(np.uint32), pos


def kuhn_mesh(n: int, seed: int = 0, jitter: float = 0.2, lo: float = -1.0, hi: float = 1.0):
    cells, pos = kuhn_grid((lo, lo, lo), (hi, hi, hi), n + 1, n + 1, n + 1)
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
    rng = np.random.default_rng(seed + 104729)
    while True:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if abs(d[1]) <= 0.99:
            return look_at_view(d * distance)


class Adam:
    """torch.optim.Adam's update on host arrays (beta = (0.9, 0.999), eps = 1e-8,
    bias-corrected; Optimizer.glsl:147-168), with an optional clamp of the
    parameter at zero after the step (pytests/train.py:352-356)."""

    def __init__(self, param: np.ndarray, lr: float, clamp_nonnegative: bool = False,
                 betas=(0.9, 0.999), eps: float = 1e-8):
        self.p, self.lr, self.clamp = param, lr, clamp_nonnegative
        self.b1, self.b2, self.eps = betas[0], betas[1], eps
        self.m = np.zeros_like(param)
        self.v = np.zeros_like(param)
        self.t = 0

    def step(self, grad: np.ndarray) -> None:
        self.t += 1
        self.m *= self.b1
        self.m += (1.0 - self.b1) * grad
        self.v *= self.b2
        self.v += (1.0 - self.b2) * grad * grad
        bc1 = 1.0 - self.b1 ** self.t
        bc2 = 1.0 - self.b2 ** self.t
        self.p -= (self.lr / bc1) * self.m / (np.sqrt(self.v / bc2) + self.eps)
        if self.clamp:
            np.maximum(self.p, 0.0, out=self.p)
