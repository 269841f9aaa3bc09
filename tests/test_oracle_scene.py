"""The oracle-side synthetic inputs (oracle/scene.py, used by the timed CPU
implementation so that it loads no product code) equal the product's
(difftetvr_b200.synthetic) bit for bit; the host Adam equals torch.optim.Adam."""
import numpy as np
import pytest
import torch

import scene as OS
from difftetvr_b200 import synthetic as S


@pytest.mark.parametrize("n,seed", [(2, 0), (8, 3), (17, 5)])
def test_kuhn_mesh_and_colours_match_product(n, seed):
    c_o, p_o = OS.kuhn_mesh(n, seed=seed)
    c_p, p_p = S.kuhn_mesh(n, seed=seed)
    assert c_o.dtype == c_p.dtype and np.array_equal(c_o, c_p)
    assert p_o.dtype == p_p.dtype and np.array_equal(p_o.view(np.uint32), p_p.view(np.uint32))
    assert np.array_equal(OS.gaussian_colors(p_o, seed=seed).view(np.uint32),
                          S.gaussian_colors(p_p, seed=seed).view(np.uint32))


def test_cameras_match_product():
    for s in (0, 100, 115, 12345):
        assert OS.sphere_camera(s) == S.sphere_camera(s)
    assert OS.FOVY_45 == S.FOVY_45


def test_host_adam_matches_torch():
    rng = np.random.default_rng(0)
    p0 = rng.normal(size=(50, 4)).astype(np.float32)
    grads = [rng.normal(size=(50, 4)).astype(np.float32) for _ in range(5)]
    p = p0.copy()
    opt = OS.Adam(p, lr=1e-2, clamp_nonnegative=True)
    t = torch.tensor(p0, requires_grad=True)
    topt = torch.optim.Adam([t], lr=1e-2)
    for g in grads:
        opt.step(g)
        t.grad = torch.tensor(g)
        topt.step()
        with torch.no_grad():
            t.clamp_(min=0.0)
    assert np.abs(p - t.detach().numpy()).max() < 1e-6
