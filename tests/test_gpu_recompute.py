"""Differentiation under a fragment budget (B200): a render whose lists exceed
the budget runs in row bands and the adjoint rebuilds each band's lists.
Images and per-pixel state equal the stored-list render bit for bit; gradients
equal it up to float-atomic summation order, and match the FP64 oracle."""
import numpy as np
import pytest
import torch

from helpers import Scene, rel_err

pytestmark = pytest.mark.gpu


def _render_and_grads(r, mesh, w):
    img = r.render().clone()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(w)
    torch.cuda.synchronize()
    return img, r.get_pixel_state(), pos.grad.clone(), col.grad.clone()


@pytest.mark.parametrize("ert", [False, True])
def test_banded_render_equals_stored(ert):
    from difftetvr_b200._lib import DTV_ERR_STATE, DtvError
    sc = Scene(16, 256, seed=3, attenuation=4.0 if ert else 1.0, ert=ert)
    mesh, r = sc.make_renderer()
    w = torch.randn(256, 256, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(2))
    img_s, (tf_s, term_s), gp_s, gc_s = _render_and_grads(r, mesh, w)
    nf = r.get_num_fragments()
    assert r.get_num_bands() == 0
    r.set_fragment_budget_bytes(nf * 8 // 6)
    img_b, (tf_b, term_b), gp_b, gc_b = _render_and_grads(r, mesh, w)
    assert r.get_num_bands() >= 6
    assert r.get_num_fragments() == nf
    assert torch.equal(img_b, img_s)
    assert np.array_equal(tf_b, tf_s) and np.array_equal(term_b, term_s)
    # Float atomics add in arrival order: equal up to summation order.
    assert rel_err(gp_b.cpu().numpy(), gp_s.cpu().numpy()) < 1e-5
    assert rel_err(gc_b.cpu().numpy(), gc_s.cpu().numpy()) < 1e-5
    with pytest.raises(DtvError) as e:
        r.get_fragment_lists()
    assert e.value.code == DTV_ERR_STATE
    # Back to stored lists when the budget allows them.
    r.set_fragment_budget_bytes(0)
    img_c = r.render()
    assert r.get_num_bands() == 0 and torch.equal(img_c, img_s)


def test_row_over_budget_raises_and_recovers():
    from difftetvr_b200._lib import DTV_ERR_BUDGET, DtvError
    sc = Scene(8, 128, seed=1)
    mesh, r = sc.make_renderer()
    r.set_fragment_budget_bytes(64)  # 8 records: less than one covered row
    with pytest.raises(DtvError) as e:
        r.render()
    assert e.value.code == DTV_ERR_BUDGET
    r.set_fragment_budget_bytes(0)
    img = r.render()
    assert r.get_num_fragments() > 0 and float(img[..., 3].max()) > 0


def test_autograd_under_budget_matches_fp64_oracle(oracle):
    """DifferentiableRenderer (autograd.Function) with banded recomputation:
    gradients of a weighted image sum vs the FP64 oracle adjoint."""
    import difftetvr_b200 as d
    sc = Scene(8, 128, seed=21)
    mesh, r = sc.make_renderer()
    r.render()
    r.set_fragment_budget_bytes(r.get_num_fragments() * 8 // 4)
    w = np.random.default_rng(4).normal(size=(128, 128, 4))
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    img = d.DifferentiableRenderer(r)()
    (img * torch.from_numpy(w.astype(np.float32)).cuda()).sum().backward()
    assert r.get_num_bands() >= 4
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    gp_o, gc_o = oracle.adjoint(fa, sc.pos, sc.col, sc.oracle_camera(oracle), sc.oracle_params(oracle), w)
    assert rel_err(pos.grad.cpu().numpy(), gp_o) < 1e-4
    assert rel_err(col.grad.cpu().numpy(), gc_o) < 1e-4
