"""Reference-facing Renderer calls beyond render / render_adjoint (B200): the
fragment-list exports (Module.cpp:960-981), reuse_intermediate_buffers_from
(Module.cpp:888-899) and set_early_ray_out_alpha (Module.cpp:869-870)."""
import numpy as np
import pytest
import torch

from helpers import Scene

pytestmark = pytest.mark.gpu


def test_fragment_exports_agree_with_the_lists():
    sc = Scene(8, 128, seed=51)
    mesh, r = sc.make_renderer()
    r.set_export_linked_list_data()
    r.render()
    torch.cuda.synchronize()
    off, rec = r.get_fragment_lists()
    assert rec.shape[0] == r.get_num_fragments() > 1000
    np.testing.assert_array_equal(r.get_fragment_buffer().numpy().view(np.uint64), rec)
    np.testing.assert_array_equal(r.get_start_offset_buffer().numpy().view(np.uint64), off)
    nodes, heads = r.get_linked_list_buffers()
    nodes = nodes.numpy().view(np.uint32)
    heads = heads.numpy().reshape(-1)
    assert nodes.shape == (rec.shape[0], 3)
    counts = np.diff(off.astype(np.int64))
    for p in np.flatnonzero(counts)[::37]:
        i, seen = int(heads[p]), []
        while i != -1:
            seen.append(i)
            i = int(nodes[i, 2].view(np.int32))
        assert seen == list(range(int(off[p]), int(off[p + 1])))
        depth = nodes[seen, 1].view(np.float32)
        assert np.all(np.diff(depth) >= 0)  # front to back
    assert (heads[counts == 0] == -1).all()


def test_reuse_intermediate_buffers_from():
    """A renderer that borrows another's fragment storage renders its own
    view exactly as a renderer with its own storage; the lender still renders
    correctly afterwards."""
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    sc = Scene(8, 128, seed=52)
    mesh, a = sc.make_renderer()
    ref_a = a.render().clone()
    b = d.Renderer(d.RendererType.PPLL)
    b.set_tet_mesh(mesh)
    b.set_viewport_size(96, 80)
    b.set_camera_fovy(S.FOVY_45)
    b.set_view_matrix(S.sphere_camera(9))
    c = d.Renderer(d.RendererType.PPLL)
    c.set_tet_mesh(mesh)
    c.set_viewport_size(96, 80)
    c.set_camera_fovy(S.FOVY_45)
    c.set_view_matrix(S.sphere_camera(9))
    ref_b = c.render().clone()
    b.reuse_intermediate_buffers_from(a)
    img_b = b.render().clone()
    torch.cuda.synchronize()
    assert img_b.shape == (80, 96, 4)
    assert torch.equal(img_b, ref_b)
    assert torch.equal(a.render(), ref_a)


def test_early_ray_out_alpha_is_one_minus_threshold():
    sc = Scene(8, 128, seed=53, attenuation=4.0, ert=True)
    mesh, r = sc.make_renderer()
    r.set_early_ray_out_thresh(0.05)
    img_t = r.render().clone()
    term_t = r.get_pixel_state()[1].copy()
    r.set_early_ray_out_alpha(0.95)
    img_a = r.render().clone()
    term_a = r.get_pixel_state()[1].copy()
    assert torch.equal(img_t, img_a) and np.array_equal(term_t, term_a)
    r.set_use_early_ray_termination(False)
    r.render()
    term_full = r.get_pixel_state()[1]
    assert (term_a < term_full).sum() > 100  # the threshold did terminate rays early
