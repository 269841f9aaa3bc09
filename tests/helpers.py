"""Shared test helpers: synthetic scenes and the product <-> oracle plumbing."""
from __future__ import annotations

import numpy as np

from difftetvr_b200 import synthetic as S


class Scene:
    def __init__(self, n: int, res: int, seed: int = 1, attenuation: float = 1.0, ert: bool = False,
                 clear=(0.0, 0.0, 0.0, 0.0), camera_seed: int | None = None, jitter: float = 0.2):
        self.n, self.res, self.seed = n, res, seed
        self.cells, self.pos = S.kuhn_mesh(n, seed=seed, jitter=jitter)
        self.col = S.gaussian_colors(self.pos, seed=seed)
        self.view = S.sphere_camera(seed if camera_seed is None else camera_seed)
        self.fovy = S.FOVY_45
        self.attenuation = attenuation
        self.ert = ert
        self.clear = clear

    def oracle_camera(self, O):
        return O.make_camera(self.view, self.fovy, self.res, self.res)

    def oracle_params(self, O, **kw):
        return O.make_params(attenuation=self.attenuation, use_ert=self.ert, clear=self.clear, **kw)

    def make_renderer(self, renderer_type=None):
        import difftetvr_b200 as d
        mesh = d.TetMesh()
        mesh.set_use_gradients(True)
        mesh.set_tet_mesh_data(self.cells, self.pos, self.col)
        r = d.Renderer(d.RendererType.PPLL if renderer_type is None else renderer_type)
        r.set_tet_mesh(mesh)
        r.set_viewport_size(self.res, self.res)
        r.set_camera_fovy(self.fovy)
        r.set_view_matrix(self.view)
        r.set_attenuation(self.attenuation)
        r.set_use_early_ray_termination(self.ert)
        r.set_clear_color(d.vec4(*self.clear))
        return mesh, r


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b||."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def two_block_scene(n: int, res: int, seed: int = 1, attenuation: float = 1.0, ert: bool = False):
    """Two disjoint jittered cubes on the diagonal, [-1, -0.2]^3 and [0.2, 1]^3,
    seen roughly along the diagonal: pixel rays cross both, so they hold two
    boundary intervals separated by empty space."""
    c1, p1 = S.kuhn_mesh(n, seed=seed, lo=-1.0, hi=-0.2)
    c2, p2 = S.kuhn_mesh(n, seed=seed + 1, lo=0.2, hi=1.0)
    sc = Scene(n, res, seed=seed, attenuation=attenuation, ert=ert)
    sc.cells = np.concatenate([c1, c2 + np.uint32(p1.shape[0])]).astype(np.uint32)
    sc.pos = np.concatenate([p1, p2]).astype(np.float32)
    sc.col = S.gaussian_colors(sc.pos, seed=seed)
    sc.view = S.look_at_view([2.3, 2.1, 2.5])
    return sc
