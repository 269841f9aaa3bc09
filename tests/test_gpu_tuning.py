"""Kernel configurations and the autotuner (B200): every tile shape and sort
method gives the same sorted lists, the same image bit for bit and the same
gradients up to float-atomic order; the autotuner leaves a valid, cached
configuration set."""
import numpy as np
import pytest
import torch

from helpers import Scene, rel_err

pytestmark = pytest.mark.gpu

CONFIGS = [dict(composite_tile=1, adjoint_tile=2, sort_surrogate_classes=0x00, sort_bucket_classes=0x00),
           dict(composite_tile=2, adjoint_tile=1, sort_surrogate_classes=0x0a, sort_bucket_classes=0x00),
           dict(composite_tile=0, adjoint_tile=0, sort_surrogate_classes=0x1e, sort_bucket_classes=0x00),
           dict(composite_tile=1, adjoint_tile=0, sort_surrogate_classes=0x00, sort_bucket_classes=0x1e),
           dict(composite_tile=0, adjoint_tile=1, sort_surrogate_classes=0x06, sort_bucket_classes=0x12)]
DEFAULT = dict(composite_tile=0, adjoint_tile=0, sort_surrogate_classes=0x1e, sort_bucket_classes=0x3c)


def _run(mesh, r, w):
    img = r.render().clone()
    off, rec = r.get_fragment_lists()
    gp = torch.zeros_like(mesh.get_vertex_positions().detach())
    gc = torch.zeros_like(mesh.get_vertex_colors().detach())
    r.render_adjoint_into(w, gp, gc)
    torch.cuda.synchronize()
    return img, off, rec, gp.cpu().numpy(), gc.cpu().numpy()


def test_every_configuration_gives_the_same_results():
    sc = Scene(16, 200, seed=6, ert=True, attenuation=3.0)
    mesh, r = sc.make_renderer()
    w = torch.randn(200, 200, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    ref = _run(mesh, r, w)
    assert r.get_tuning() == DEFAULT
    for cfg in CONFIGS:
        r.set_tuning(**cfg)
        assert r.get_tuning() == cfg
        img, off, rec, gp, gc = _run(mesh, r, w)
        assert torch.equal(img, ref[0])
        assert np.array_equal(off, ref[1]) and np.array_equal(rec, ref[2])
        assert rel_err(gp, ref[3]) < 1e-5 and rel_err(gc, ref[4]) < 1e-5
    with pytest.raises(RuntimeError):
        r.set_tuning(composite_tile=3)
    with pytest.raises(RuntimeError):
        r.set_tuning(sort_surrogate_classes=0x1)
    with pytest.raises(RuntimeError):
        r.set_tuning(sort_bucket_classes=0x40)


def test_autotuner_sets_and_caches_a_configuration():
    from difftetvr_b200 import autotune
    sc = Scene(12, 160, seed=3)
    mesh, r = sc.make_renderer()
    out = autotune.autotune_renderer(r, trials=2, force=True)
    t = out["tuning"]
    assert t["composite_tile"] in (0, 1, 2) and t["adjoint_tile"] in (0, 1, 2)
    assert (t["sort_surrogate_classes"] & ~0x1e) == 0 and (t["sort_bucket_classes"] & ~0x3e) == 0
    assert r.get_tuning() == t and len(out["timings"]) >= 14 and out["ms"] > 0
    r.set_tuning(composite_tile=(t["composite_tile"] + 1) % 3)
    again = autotune.autotune_renderer(r)  # cached: restores the chosen configuration
    assert again is out and r.get_tuning() == t


def test_batch_sort_configuration_and_autotune():
    import difftetvr_b200 as d
    from difftetvr_b200 import autotune
    from difftetvr_b200 import synthetic as S
    from difftetvr_b200.batch import BatchRenderer, View
    meshes = []
    for n, seed in ((10, 1), (6, 2)):
        cells, pos = S.kuhn_mesh(n, seed=seed)
        m = d.TetMesh()
        m.set_use_gradients(True)
        m.set_tet_mesh_data(cells, pos, S.gaussian_colors(pos, seed=seed))
        meshes.append(m)
    br = BatchRenderer(meshes, attenuation=1.0)
    views = [View(mesh=i % 2, view_matrix=S.sphere_camera(50 + i), width=96, height=80) for i in range(4)]
    ref = [im.clone() for im in br.render(views)]
    for q, b in ((0x00, 0x00), (0x14, 0x00), (0x00, 0x1e)):
        br.set_tuning(sort_surrogate_classes=q, sort_bucket_classes=b)
        assert br.get_tuning() == dict(sort_surrogate_classes=q, sort_bucket_classes=b)
        for a, b in zip(br.render(views), ref):
            assert torch.equal(a, b)
    out = autotune.autotune_batch(br, views, trials=1, force=True)
    assert br.get_tuning() == out["tuning"] and len(out["timings"]) == 10  # 1 + 4 classes x 2 + class 5 x 1
