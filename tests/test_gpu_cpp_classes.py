"""The C++ classes of include/difftetvr_b200.hpp (TetMesh / Renderer over the C
ABI, the reference's C++ interface names) against the Python path: one render
+ adjoint of the same mesh, view and image adjoint through the compiled check
program (tests/cpp/cabi_classes.cpp) give the same image and gradients."""
import os
import subprocess

import numpy as np
import pytest
import torch

from helpers import Scene, rel_err
from test_cabi import load_cpp_build

pytestmark = pytest.mark.gpu


def test_cpp_renderer_matches_python(tmp_path):
    res = 128
    sc = Scene(8, res, seed=21)
    w = np.random.default_rng(21).normal(size=(res, res, 4)).astype(np.float32)
    d = str(tmp_path)
    sc.cells.astype(np.uint32).tofile(os.path.join(d, "cells.u32"))
    sc.pos.astype(np.float32).tofile(os.path.join(d, "pos.f32"))
    sc.col.astype(np.float32).tofile(os.path.join(d, "col.f32"))
    np.asarray(sc.view, np.float32).tofile(os.path.join(d, "view.f32"))
    w.tofile(os.path.join(d, "adj.f32"))
    exe = load_cpp_build().build()
    out = subprocess.run([exe, "render", d, str(res)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "OK render" in out.stdout
    img_c = np.fromfile(os.path.join(d, "image.f32"), np.float32).reshape(res, res, 4)
    gp_c = np.fromfile(os.path.join(d, "gpos.f32"), np.float32).reshape(-1, 3)
    gc_c = np.fromfile(os.path.join(d, "gcol.f32"), np.float32).reshape(-1, 4)

    mesh, r = sc.make_renderer()
    img = r.render().cpu().numpy()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda())
    assert np.array_equal(img_c, img)  # same kernels, same inputs
    assert (img[..., 3] > 0).sum() > 1000
    # Float atomics accumulate in a run-dependent order.
    assert rel_err(gp_c, pos.grad.cpu().numpy()) < 1e-5
    assert rel_err(gc_c, col.grad.cpu().numpy()) < 1e-5
