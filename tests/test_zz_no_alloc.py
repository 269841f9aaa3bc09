"""dtv_render_noalloc, the allocation-free forward render for callers that
cannot allocate device memory while rendering, against dtv_renderer_render.

Collected last (file name) so a failure here leaves every other test run."""
import ctypes

import numpy as np
import pytest
import torch

from difftetvr_b200 import _lib
from difftetvr_b200 import synthetic as S
from helpers import Scene

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5


def _noalloc_render(mesh, renderer, positions, colors):
    """Call the C ABI entry point with the renderer's camera and settings."""
    cam = renderer._camera()
    prm = renderer._params()
    image = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=positions.device)
    _lib.call("dtv_render_noalloc", mesh.native.handle, positions.data_ptr(), colors.data_ptr(), ctypes.byref(cam),
              ctypes.byref(prm), image.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return image


def test_noalloc_matches_renderer_on_two_calls_in_a_row():
    sc = Scene(8, 128, seed=31)
    mesh, r = sc.make_renderer()
    pos = mesh.get_vertex_positions().detach()
    col = mesh.get_vertex_colors().detach()

    # Call 1: the scene's camera.
    ref1 = r.render().clone()
    out1 = _noalloc_render(mesh, r, pos, col)
    torch.cuda.synchronize()
    assert torch.isfinite(out1).all()
    assert (ref1[..., 3] > 0).sum() > 1000
    assert float((out1 - ref1).abs().max()) <= IMG_TOL

    # Call 2, right after: another camera and other colours, with early ray
    # termination on; the scratch keeps call 1's contents and must not leak.
    r.set_view_matrix(S.sphere_camera(77))
    r.set_use_early_ray_termination(True)
    r.set_attenuation(3.0)
    col2 = (col * torch.tensor([0.5, 1.0, 0.25, 2.0], device=col.device)).contiguous()
    mesh._colors.data.copy_(col2)
    ref2 = r.render().clone()
    out2 = _noalloc_render(mesh, r, pos, col2)
    torch.cuda.synchronize()
    assert float((out2 - ref2).abs().max()) <= IMG_TOL
    assert float((out2 - out1).abs().max()) > 1e-3  # really a different image


def test_noalloc_rejects_sizes_beyond_its_limits():
    sc = Scene(4, 300, seed=2)  # 300 x 300 = 90,000 pixels > 65,536
    mesh, r = sc.make_renderer()
    pos = mesh.get_vertex_positions().detach()
    col = mesh.get_vertex_colors().detach()
    with pytest.raises(_lib.DtvError) as e:
        _noalloc_render(mesh, r, pos, col)
    assert e.value.code == _lib.DTV_ERR_ARG
    assert "pixels exceed" in str(e.value)
    # A valid call still works after the rejection.
    r.set_viewport_size(64, 64)
    ref = r.render().clone()
    out = _noalloc_render(mesh, r, pos, col)
    torch.cuda.synchronize()
    assert float((out - ref).abs().max()) <= IMG_TOL
    assert np.isfinite(out.cpu().numpy()).all()


def test_noalloc_fragment_and_vertex_limits_then_valid_call():
    """The fragment limit (4,194,304 records) is checked after the exact count
    of the scan, once the per-pixel counters are written; the budget of the
    call's parameters likewise.  The next valid call must clear what the
    rejected one left and match dtv_renderer_render."""
    from difftetvr_b200._lib import DTV_ERR_ARG, DTV_ERR_BUDGET
    sc = Scene(32, 256, seed=3)  # 35,937 vertices, about 6.4 M fragments at 256 x 256
    mesh, r = sc.make_renderer()
    pos = mesh.get_vertex_positions().detach()
    col = mesh.get_vertex_colors().detach()
    with pytest.raises(_lib.DtvError) as e:
        _noalloc_render(mesh, r, pos, col)
    assert e.value.code == DTV_ERR_BUDGET and "fragments exceed" in str(e.value)
    r.set_viewport_size(128, 128)
    ref = r.render().clone()
    out = _noalloc_render(mesh, r, pos, col)
    torch.cuda.synchronize()
    assert float((out - ref).abs().max()) <= IMG_TOL

    # The caller's own fragment budget, then a valid call again.
    r.set_fragment_budget_bytes(1024)
    with pytest.raises(_lib.DtvError) as e:
        _noalloc_render(mesh, r, pos, col)
    assert e.value.code == DTV_ERR_BUDGET and "fragment_budget_bytes" in str(e.value)
    r.set_fragment_budget_bytes(0)
    out = _noalloc_render(mesh, r, pos, col)
    torch.cuda.synchronize()
    assert float((out - ref).abs().max()) <= IMG_TOL

    # Vertex limit (65,536): a 40^3 mesh has 68,921 vertices.
    big = Scene(40, 64, seed=4)
    mesh_b, r_b = big.make_renderer()
    with pytest.raises(_lib.DtvError) as e:
        _noalloc_render(mesh_b, r_b, mesh_b.get_vertex_positions().detach(), mesh_b.get_vertex_colors().detach())
    assert e.value.code == DTV_ERR_ARG and "vertices exceed" in str(e.value)
