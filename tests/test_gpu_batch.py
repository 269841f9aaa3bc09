"""Batched multi-view / multi-mesh path vs the per-view plain path (B200)."""
import numpy as np
import pytest
import torch

import difftetvr_b200 as d
from difftetvr_b200 import synthetic as S
from difftetvr_b200.batch import BatchRenderer, View
from difftetvr_b200.optim import CLAMP_NONNEGATIVE, Adam, l2_loss
from helpers import rel_err

pytestmark = pytest.mark.gpu


def make_mesh(n, seed):
    cells, pos = S.kuhn_mesh(n, seed=seed)
    col = S.gaussian_colors(pos, seed=seed)
    m = d.TetMesh()
    m.set_use_gradients(True)
    m.set_tet_mesh_data(cells, pos, col)
    return m


def plain_renderer(mesh, v: View, attenuation=1.0, ert=True):
    r = d.Renderer(d.RendererType.PPLL)
    r.set_tet_mesh(mesh)
    r.set_viewport_size(v.width, v.height)
    r.set_camera_fovy(v.fovy)
    r.set_view_matrix(v.view_matrix)
    r.set_attenuation(attenuation)
    r.set_use_early_ray_termination(ert)
    r.set_clear_color(d.vec4(0, 0, 0, 0))
    return r


def views_for(meshes_idx, sizes):
    return [View(mesh=m, view_matrix=S.sphere_camera(40 + i), width=w, height=h)
            for i, (m, (w, h)) in enumerate(zip(meshes_idx, sizes))]


def test_batch_render_matches_plain_views():
    meshes = [make_mesh(8, 1), make_mesh(6, 2), make_mesh(10, 3)]
    br = BatchRenderer(meshes, attenuation=1.0)
    views = views_for([0, 1, 2, 0, 2], [(64, 64), (96, 80), (128, 128), (40, 72), (17, 33)])
    imgs = br.render(views)
    torch.cuda.synchronize()
    for v, img in zip(views, imgs):
        ref = plain_renderer(meshes[v.mesh], v).render()
        assert float((img - ref).abs().max()) <= 1e-6


def test_batch_wide_faces_match_plain_views():
    """Meshes of 1 and 2 cubes per axis at 512^2: face boxes over 64 px take the
    64-bit raster path (listed by the count), beside an ordinary 8^3 view."""
    meshes = [make_mesh(1, 6), make_mesh(2, 7), make_mesh(8, 8)]
    br = BatchRenderer(meshes, attenuation=1.0)
    views = views_for([0, 1, 2, 1], [(512, 512), (512, 384), (96, 96), (300, 512)])
    imgs = br.render(views)
    torch.cuda.synchronize()
    nf = 0
    for v, img in zip(views, imgs):
        r = plain_renderer(meshes[v.mesh], v)
        ref = r.render()
        nf += r.get_num_fragments()
        assert float((img - ref).abs().max()) <= 1e-6
    assert br.info()["fragments"] == nf


def test_batch_adjoint_matches_sum_of_plain_adjoints():
    meshes = [make_mesh(8, 4), make_mesh(6, 5)]
    br = BatchRenderer(meshes, attenuation=2.0)
    views = views_for([0, 1, 0, 1], [(64, 64), (80, 48), (96, 96), (32, 32)])
    g = torch.Generator(device="cuda").manual_seed(0)
    for i, v in enumerate(views):
        v.image_adjoint = torch.randn(v.height, v.width, 4, device="cuda", generator=g)
        v.grad_slot = v.mesh
    br.render(views)
    slots = [(m, torch.zeros_like(meshes[m].get_vertex_positions()), torch.zeros_like(meshes[m].get_vertex_colors()))
             for m in range(2)]
    br.render_adjoint(slots)
    torch.cuda.synchronize()
    for m in range(2):
        gp = torch.zeros_like(meshes[m].get_vertex_positions())
        gc = torch.zeros_like(meshes[m].get_vertex_colors())
        for v in views:
            if v.mesh != m:
                continue
            meshes[m].get_vertex_positions().grad.zero_()
            meshes[m].get_vertex_colors().grad.zero_()
            r = plain_renderer(meshes[m], v, attenuation=2.0)
            r.render()
            r.render_adjoint(v.image_adjoint)
            gp += meshes[m].get_vertex_positions().grad
            gc += meshes[m].get_vertex_colors().grad
        assert rel_err(slots[m][1].cpu().numpy(), gp.cpu().numpy()) < 1e-5
        assert rel_err(slots[m][2].cpu().numpy(), gc.cpu().numpy()) < 1e-5


def _targets(meshes_idx, views, seed=9):
    """Target images rendered from different-seed meshes of the same topology."""
    tm = {m: make_mesh(n, seed + m) for m, n in meshes_idx.items()}
    for v in views:
        v.target = plain_renderer(tm[v.mesh], v).render().clone()


def _plain_step(meshes, views, opts):
    for m, o in zip(meshes, opts):
        o.zero_grad(set_to_none=False)
    total = 0.0
    for v in views:
        r = plain_renderer(meshes[v.mesh], v)
        img = d.DifferentiableRenderer(r)()
        loss = l2_loss(img, v.target)
        loss.backward()
        total += float(loss)
    for o in opts:
        o.step()
    return total


@pytest.mark.parametrize("graph", [False, True])
def test_batch_train_step_matches_plain_loop(graph):
    sizes = {0: 8, 1: 6}
    meshes_b = [make_mesh(8, 1), make_mesh(6, 2)]
    meshes_p = [make_mesh(8, 1), make_mesh(6, 2)]
    views = views_for([0, 1, 0, 1, 0], [(64, 64), (48, 48), (80, 64), (32, 48), (64, 40)])
    _targets(sizes, views)
    br = BatchRenderer(meshes_b, attenuation=1.0)
    br.set_graph(graph)
    opts = [Adam([{"params": [m.get_vertex_colors()], "lr": 1e-2, "clamp": CLAMP_NONNEGATIVE},
                  {"params": [m.get_vertex_positions()], "lr": 1e-4}]) for m in meshes_p]
    for step in range(4):
        lb = float(br.train_step(views, lr_positions=1e-4, lr_colors=1e-2, clamp_colors=1))
        lp = _plain_step(meshes_p, views, opts)
        assert abs(lb - lp) <= 1e-5 * max(1.0, abs(lp))
    torch.cuda.synchronize()
    for mb, mp in zip(meshes_b, meshes_p):
        assert rel_err(mb.get_vertex_positions().detach().cpu().numpy(),
                       mp.get_vertex_positions().detach().cpu().numpy()) < 1e-6
        assert rel_err(mb.get_vertex_colors().detach().cpu().numpy(),
                       mp.get_vertex_colors().detach().cpu().numpy()) < 1e-5
    info = br.info()
    assert info["graph"] == graph and info["fragments"] > 0


def test_batch_graph_overflow_reruns_step_exactly():
    """Growing the views after the graph was captured overflows the record
    buffer: the step is rerun uncaptured with a larger buffer and the result
    equals an eager batch."""
    views_small = views_for([0, 0], [(48, 48), (48, 48)])
    views_big = views_for([0, 0], [(128, 128), (128, 128)])
    _targets({0: 8}, views_small + views_big)
    res = []
    for graph in (True, False):
        m = make_mesh(8, 1)
        br = BatchRenderer([m], attenuation=1.0)
        br.set_graph(graph)
        for _ in range(2):
            br.train_step(views_small)
        br.train_step(views_big)
        br.train_step(views_big)
        torch.cuda.synchronize()
        res.append((m.get_vertex_colors().detach().cpu().numpy(), br.info()))
    assert res[0][1]["steps_rerun"] >= 1
    assert np.abs(res[0][0] - res[1][0]).max() < 1e-6
