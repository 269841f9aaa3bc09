"""Serving on the B200: every result of a mixed request stream equals the same
request rendered alone through the plain path."""
import math

import pytest
import torch

import difftetvr_b200 as d
from difftetvr_b200 import synthetic as S
from difftetvr_b200.serve import GpuBackend, Request, ServingEngine
from helpers import rel_err

pytestmark = pytest.mark.gpu


def make_mesh(n, seed):
    cells, pos = S.kuhn_mesh(n, seed=seed)
    m = d.TetMesh()
    m.set_use_gradients(True)
    m.set_tet_mesh_data(cells, pos, S.gaussian_colors(pos, seed=seed))
    return m


def alone(mesh, r: Request):
    rd = d.Renderer(d.RendererType.PPLL)
    rd.set_tet_mesh(mesh)
    rd.set_viewport_size(r.width, r.height)
    rd.set_camera_fovy(r.fovy)
    rd.set_view_matrix(r.view_matrix)
    rd.set_attenuation(1.0)
    rd.set_use_early_ray_termination(True)
    img = rd.render().clone()
    gp = gc = None
    if r.mode == "gradient":
        mesh.get_vertex_positions().grad.zero_()
        mesh.get_vertex_colors().grad.zero_()
        rd.render_adjoint(((img - r.target) * (2.0 / img.numel())).contiguous())
        gp = mesh.get_vertex_positions().grad.clone()
        gc = mesh.get_vertex_colors().grad.clone()
    return img, gp, gc


def test_mixed_stream_results_equal_isolated_results():
    meshes = {"a": make_mesh(8, 1), "b": make_mesh(6, 2), "c": make_mesh(10, 3)}
    be = GpuBackend(meshes, slots=2)
    be.calibrate(S.sphere_camera(0), res=64)
    eng = ServingEngine(be, budget_fragments=4_000_000, max_batch=6)
    g = torch.Generator(device="cuda").manual_seed(1)
    reqs = []
    sizes = [(64, 64), (48, 80), (96, 96), (32, 32)]
    for i in range(18):
        w, h = sizes[i % len(sizes)]
        mode = "gradient" if i % 3 == 0 else "forward"
        tgt = torch.rand(h, w, 4, device="cuda", generator=g) if mode == "gradient" else None
        reqs.append(Request(mesh="abc"[i % 3], view_matrix=S.sphere_camera(100 + i), width=w, height=h,
                            mode=mode, target=tgt, fovy=math.radians(45.0)))
    torch.cuda.synchronize()
    eng.start()
    futs = [eng.submit(r) for r in reqs]
    results = [f.result(timeout=120) for f in futs]
    eng.stop()
    assert eng.batches < len(reqs)  # requests were actually batched
    for r, res in zip(reqs, results):
        img, gp, gc = alone(meshes[r.mesh], r)
        assert float((res.image - img).abs().max()) <= 1e-6
        if r.mode == "gradient":
            assert rel_err(res.grad_positions.cpu().numpy(), gp.cpu().numpy()) < 1e-5
            assert rel_err(res.grad_colors.cpu().numpy(), gc.cpu().numpy()) < 1e-5
    st = eng.latency_stats()
    assert st["requests"] == len(reqs) and st["p99_ms"] > 0


@pytest.mark.parametrize("reserve_fragments", [4_000_000, 20_000])
def test_reserved_async_serving_equals_isolated(reserve_fragments):
    """With reserved slot scratch the engine enqueues batches without a host
    synchronisation; a batch over the reserved record capacity (the small
    reservation) is detected when it completes and run again exactly."""
    meshes = {"a": make_mesh(8, 1), "b": make_mesh(6, 2)}
    be = GpuBackend(meshes, slots=2)
    be.calibrate(S.sphere_camera(0), res=64)
    be.reserve(4, 96 * 96, reserve_fragments)
    eng = ServingEngine(be, budget_fragments=4_000_000, max_batch=4)
    g = torch.Generator(device="cuda").manual_seed(2)
    reqs = []
    for i in range(10):
        mode = "gradient" if i % 2 == 0 else "forward"
        tgt = torch.rand(96, 96, 4, device="cuda", generator=g) if mode == "gradient" else None
        reqs.append(Request(mesh="ab"[i % 2], view_matrix=S.sphere_camera(200 + i), width=96, height=96,
                            mode=mode, target=tgt, fovy=math.radians(45.0)))
    torch.cuda.synchronize()
    eng.start()
    results = [f.result(timeout=120) for f in [eng.submit(r) for r in reqs]]
    eng.stop()
    for r, res in zip(reqs, results):
        img, gp, gc = alone(meshes[r.mesh], r)
        assert float((res.image - img).abs().max()) <= 1e-6
        if r.mode == "gradient":
            assert rel_err(res.grad_positions.cpu().numpy(), gp.cpu().numpy()) < 1e-5
            assert rel_err(res.grad_colors.cpu().numpy(), gc.cpu().numpy()) < 1e-5
