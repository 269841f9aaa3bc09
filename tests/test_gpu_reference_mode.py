"""Distance of the CUDA path from the reference's own formulas (the oracle's
reference mode) on the same inputs, at the plain-method configurations:
Kuhn 16^3 at 512^2 (whole image) and Kuhn 64^3 at 1024^2 (four 64-row bands of
the benchmark's first view).  The reference cannot run here (Vulkan), so its
GLSL restated in the oracle stands in for it.  The measured distances are
printed (pytest -s) and bounded:
- images: the reference's FP32 NDC depth (~5e-5 of view depth at distance 3)
  and its unsigned weights change a few pixels by up to ~1e-3;
- colour gradients: equal to the reference adjoint run over all four
  sub-segments; the reference's own loop skips the first (Backward.glsl:222);
- position gradients: the reference differentiates the Euclidean segment
  length with the world point held fixed (BackwardCommon.glsl:139-251), so
  its position gradient is not the derivative of its forward; only the
  distance is recorded."""
import numpy as np
import pytest
import torch

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _cos(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))


@pytest.mark.parametrize("n,seed,cam_seed,res,bands", [
    (16, 16, 16, 512, None),
    (64, 0, 100, 1024, (192, 448, 576, 832)),
])
def test_cuda_vs_reference_formulas(oracle, n, seed, cam_seed, res, bands):
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    cells, pos = S.kuhn_mesh(n, seed=seed)
    col = S.gaussian_colors(pos, seed=seed)
    view = S.sphere_camera(cam_seed)
    mesh = d.TetMesh()
    mesh.set_use_gradients(True)
    mesh.set_tet_mesh_data(cells, pos, col)
    r = d.Renderer(d.RendererType.PPLL)
    r.set_tet_mesh(mesh)
    r.set_viewport_size(res, res)
    r.set_camera_fovy(S.FOVY_45)
    r.set_view_matrix(view)
    r.set_attenuation(1.0)
    r.set_use_early_ray_termination(False)
    img = r.render().cpu().numpy().astype(np.float64)
    fa = oracle.Faces(cells, pos.shape[0])
    cam = oracle.make_camera(view, S.FOVY_45, res, res)
    rng = np.random.default_rng(n)
    w = np.zeros((res, res, 4))
    rows = [(0, res)] if bands is None else [(y, y + 64) for y in bands]
    img_r = np.zeros_like(img)
    gp_r = np.zeros((pos.shape[0], 3))
    gc_r = np.zeros((pos.shape[0], 4))
    gc_all = np.zeros((pos.shape[0], 4))
    mask = np.zeros((res, res), bool)
    for y0, y1 in rows:
        mask[y0:y1] = True
        w[y0:y1] = rng.standard_normal((y1 - y0, res, 4))
        prm = oracle.make_params(attenuation=1.0, rows=(y0, y1))
        i_r, _, g_p, g_c = oracle.refmode(fa, pos, col, cam, prm, w)
        img_r[y0:y1] = i_r[y0:y1]
        gp_r += g_p
        gc_r += g_c
        gc_all += oracle.refmode(fa, pos, col, cam, prm, w, skip0=False)[3]
    pos_t, col_t = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos_t.grad.zero_()
    col_t.grad.zero_()
    r.render_adjoint(torch.from_numpy(w.astype(np.float32)).cuda())
    gp = pos_t.grad.cpu().numpy()
    gc = col_t.grad.cpu().numpy()
    e = np.abs(img - img_r)[mask]
    stats = {
        "config": f"Kuhn {n}^3 at {res}^2" + ("" if bands is None else " (4 bands of 64 rows)"),
        "image_max": float(e.max()), "image_mean": float(e.mean()),
        "grad_col_rel": rel_err(gc, gc_r), "grad_col_rel_all_subsegments": rel_err(gc, gc_all),
        "grad_pos_rel": rel_err(gp, gp_r), "grad_pos_cos": _cos(gp, gp_r), "grad_col_cos": _cos(gc, gc_r),
    }
    print("\nCUDA vs reference formulas:", stats)
    assert stats["image_max"] < 5e-3 and stats["image_mean"] < 1e-4
    assert stats["grad_col_rel_all_subsegments"] < 2e-3
