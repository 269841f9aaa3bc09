"""CUDA path vs the committed FP64-oracle fixtures (B200): sorted fragment
lists bit-exact, images within 1e-5, gradients within 1e-4 relative; and
TetMesh.load_from_file / save_to_file with the .bintet fixtures."""
import hashlib
import os

import numpy as np
import pytest
import torch

from difftetvr_b200 import synthetic as S
from helpers import rel_err

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _renderer(cells, pos, col, view, res):
    import difftetvr_b200 as d
    m = d.TetMesh()
    m.set_use_gradients(True)
    m.set_tet_mesh_data(cells, pos, col)
    r = d.Renderer(d.RendererType.PPLL)
    r.set_tet_mesh(m)
    r.set_viewport_size(res, res)
    r.set_camera_fovy(S.FOVY_45)
    r.set_view_matrix(view)
    r.set_attenuation(1.0)
    r.set_use_early_ray_termination(False)
    r.set_clear_color(d.vec4(0, 0, 0, 0))
    return m, r


def _grads(m, r, seed, res):
    w = np.random.default_rng(seed).normal(size=(res, res, 4)).astype(np.float32)
    p, c = m.get_vertex_positions(), m.get_vertex_colors()
    p.grad.zero_()
    c.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda())
    return p.grad.cpu().numpy(), c.grad.cpu().numpy()


def test_matches_fixture_8_128():
    g = np.load(os.path.join(GOLDEN, "oracle_8_128.npz"))
    res = int(g["res"])
    m, r = _renderer(g["cells"], g["positions"], g["colors"], g["view"].tolist(), res)
    img = r.render().cpu().numpy().astype(np.float64)
    off, rec = r.get_fragment_lists()
    assert np.array_equal(off.astype(np.int64), g["offsets"]) and np.array_equal(rec, g["records"])
    assert np.abs(img - g["image"]).max() < 1e-5
    gp, gc = _grads(m, r, int(g["image_adjoint_seed"]), res)
    assert rel_err(gp, g["grad_positions"]) < 1e-4
    assert rel_err(gc, g["grad_colors"]) < 1e-4


def test_matches_fixture_16_512():
    g = np.load(os.path.join(GOLDEN, "oracle_16_512.npz"))
    res = int(g["res"])
    cells, pos = S.kuhn_mesh(16, seed=16, jitter=0.2)
    col = S.gaussian_colors(pos, seed=16)
    m, r = _renderer(cells, pos, col, g["view"].tolist(), res)
    img = r.render().cpu().numpy().astype(np.float64)
    off, rec = r.get_fragment_lists()
    assert np.array_equal(off.astype(np.int64), g["offsets"])
    assert hashlib.sha256(rec.tobytes()).hexdigest() == str(g["records_sha256"])
    assert r.get_num_fragments() == int(g["num_fragments"])
    assert np.abs(img.reshape(-1, 4)[g["pixels"]] - g["image_at_pixels"]).max() < 1e-5
    assert np.abs(img.sum(axis=(0, 1)) - g["image_sum"]).max() < 1e-5 * res * res
    gp, gc = _grads(m, r, int(g["image_adjoint_seed"]), res)
    assert rel_err(gp, g["grad_positions"]) < 1e-4
    assert rel_err(gc, g["grad_colors"]) < 1e-4


def test_load_and_save_bintet(tmp_path):
    import difftetvr_b200 as d
    m = d.TetMesh()
    assert m.load_from_file(os.path.join(GOLDEN, "single_tet_v1.bintet"))
    ref = d.TetMesh()
    ref.load_test_data(d.TestCase.SINGLE_TETRAHEDRON)
    assert torch.equal(m.get_vertex_positions().detach(), ref.get_vertex_positions().detach())
    assert torch.equal(m.get_vertex_colors().detach(), ref.get_vertex_colors().detach())
    out = str(tmp_path / "copy.bintet")
    assert m.save_to_file(out)
    assert open(out, "rb").read() == open(os.path.join(GOLDEN, "single_tet_v1.bintet"), "rb").read()
    with pytest.warns(UserWarning):
        assert not m.load_from_file(str(tmp_path / "mesh.vtk"))
    with pytest.raises(RuntimeError):
        m.save_to_file(str(tmp_path / "mesh.vtk"))
