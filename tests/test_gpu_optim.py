"""Loss and Adam kernels vs torch (B200)."""
import ctypes

import numpy as np
import pytest
import torch

from difftetvr_b200 import _lib

pytestmark = pytest.mark.gpu


def test_l2_loss_kernel_matches_torch():
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(64, 48, 4, device="cuda", generator=g)
    y = torch.rand(64, 48, 4, device="cuda", generator=g)
    adj = torch.empty_like(x)
    loss = torch.zeros(1, device="cuda")
    n = x.numel()
    _lib.call("dtv_loss_l2", x.data_ptr(), y.data_ptr(), n, 1.0 / n, adj.data_ptr(), loss.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    xr = x.clone().requires_grad_(True)
    ref = torch.nn.functional.mse_loss(xr, y)
    ref.backward()
    assert torch.allclose(loss[0], ref, rtol=1e-5)
    assert torch.allclose(adj, xr.grad, rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("clamp", [0, 1])
def test_adam_kernel_matches_torch_adam(clamp):
    g = torch.Generator(device="cuda").manual_seed(1)
    p0 = torch.randn(3000, device="cuda", generator=g)
    p_ref = p0.clone().requires_grad_(True)
    opt = torch.optim.Adam([p_ref], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    p = p0.clone()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    for step in range(1, 6):
        grad = torch.randn(3000, device="cuda", generator=g)
        p_ref.grad = grad.clone()
        opt.step()
        if clamp == 1:
            with torch.no_grad():
                p_ref -= torch.min(p_ref, torch.zeros_like(p_ref))
        _lib.call("dtv_adam_step", p.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                  ctypes.c_float(1e-2), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), step,
                  clamp, None, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert torch.allclose(p, p_ref.detach(), rtol=1e-5, atol=1e-6)


def test_adam_fixed_mask_modes():
    p = torch.ones(12, device="cuda")
    grad = torch.ones(12, device="cuda")
    mask = torch.tensor([1, 0, 0, 1], dtype=torch.int32, device="cuda")  # per vertex (stride 3)
    for mode in (1, 2):
        q = p.clone()
        m = torch.zeros_like(q)
        v = torch.zeros_like(q)
        _lib.call("dtv_adam_step", q.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), 12,
                  ctypes.c_float(0.1), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), 1, 0,
                  mask.data_ptr(), mode, 3, torch.cuda.current_stream().cuda_stream)
        fixed = mask.repeat_interleave(3).bool()
        assert torch.all(q[fixed] == 1.0)
        assert torch.all(q[~fixed] < 1.0)
        if mode == 2:
            assert torch.all(m[fixed] == 0)
