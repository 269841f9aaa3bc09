"""CUDA tet-quality regularizer vs the FP64 oracle (B200), and its use in the
autograd path (DifferentiableRenderer with use_tet_regularizer, the
reference's pytests/pyutils.py:45-46 order: regularizer, then adjoint)."""
import numpy as np
import pytest
import torch

from difftetvr_b200 import synthetic as S
from helpers import Scene, rel_err

pytestmark = pytest.mark.gpu


def _mesh(cells, pos, col=None):
    import difftetvr_b200 as d
    m = d.TetMesh()
    m.set_use_gradients(True)
    m.set_tet_mesh_data(cells, pos, S.gaussian_colors(pos, seed=1) if col is None else col)
    return m


@pytest.mark.parametrize("n,perturb", [(8, True), (16, False), (64, False)])
def test_gradient_and_penalty_match_fp64_oracle(oracle, n, perturb):
    """8^3 with an interior vertex pushed to invert cells; 16^3; 64^3, whose
    small tets fall under the reference's denominator clamp."""
    import difftetvr_b200 as d
    cells, pos = S.kuhn_mesh(n, seed=n, jitter=0.3)
    if perturb:
        v = (n // 2) * ((n + 1) ** 2 + (n + 1) + 1)
        pos[v] += np.array([0.35, -0.3, 0.4], np.float32) * (2.0 / n)
    m = _mesh(cells, pos)
    reg = d.TetRegularizer(m, 0.3, 5.0)
    g = torch.zeros(pos.shape[0], 3, device="cuda")
    loss = reg.compute_grad_into(g)
    total_o, g_o = oracle.tet_regularizer(cells, pos.astype(np.float64), 0.3, 5.0)
    assert rel_err(g.cpu().numpy(), g_o) < 1e-5, rel_err(g.cpu().numpy(), g_o)
    assert abs(float(loss) - total_o) <= 1e-5 * abs(total_o)
    # compute_grad adds into .grad
    p = m.get_vertex_positions()
    p.grad.zero_()
    reg.compute_grad()
    reg.compute_grad()
    assert rel_err(p.grad.cpu().numpy(), 2 * g_o) < 1e-5


def test_autograd_with_regularizer_adds_both_gradients():
    import difftetvr_b200 as d
    sc = Scene(8, 96, seed=5)
    mesh, r = sc.make_renderer()
    w = torch.randn(96, 96, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    p, c = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    p.grad.zero_()
    c.grad.zero_()
    (d.DifferentiableRenderer(r)() * w).sum().backward()
    g_render = p.grad.clone()
    p.grad.zero_()
    c.grad.zero_()
    dr = d.DifferentiableRenderer(r, use_tet_regularizer=True, tet_reg_lambda=0.5, tet_reg_softplus_beta=3.0)
    (dr() * w).sum().backward()
    g_reg = torch.zeros_like(g_render)
    d.TetRegularizer(mesh, 0.5, 3.0).compute_grad_into(g_reg)
    torch.cuda.synchronize()
    assert rel_err(p.grad.cpu().numpy(), (g_render + g_reg).cpu().numpy()) < 1e-5
