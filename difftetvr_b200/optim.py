"""Fused Adam and L2 loss on the CUDA library.

``Adam`` is a torch.optim.Optimizer whose step runs one kernel per parameter
tensor (the update of Optimizer.glsl:88-169 / torch.optim.Adam as used by
pytests/train.py:318, with the colour clamp of train.py:352-356 and the
boundary freeze of train.py:349-350 as options).  ``l2_loss`` is
torch.nn.MSELoss(reduction='mean') with the loss value and the image adjoint
produced by one kernel (Loss.glsl:242-248).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

CLAMP_NONE = 0
CLAMP_NONNEGATIVE = 1   # p = max(p, 0)            (train.py:352-356)
CLAMP_RGBA = 2          # rgb in [0,1], alpha >= 0  (Optimizer.glsl:161-167)


class Adam(torch.optim.Optimizer):
    """Per-group options: lr, betas, eps, clamp (CLAMP_*), fixed_mask (int32 per
    group of `stride` values, e.g. vertex boundary bits), fixed_mode (1 = zero
    gradient, 2 = skip update), stride."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, clamp=CLAMP_NONE, fixed_mask=None,
                 fixed_mode=0, stride=1):
        defaults = dict(lr=lr, betas=betas, eps=eps, clamp=clamp, fixed_mask=fixed_mask, fixed_mode=fixed_mode,
                        stride=stride)
        super().__init__(params, defaults)

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        for group in self.param_groups:
            b1, b2 = group["betas"]
            mask = group["fixed_mask"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                if p.dtype != torch.float32 or not p.is_cuda or not p.is_contiguous():
                    raise RuntimeError("difftetvr_b200.optim.Adam needs contiguous float32 CUDA tensors")
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p)
                    st["exp_avg_sq"] = torch.zeros_like(p)
                st["step"] += 1
                grad = p.grad.contiguous()
                _lib.call("dtv_adam_step", p.data_ptr(), grad.data_ptr(), st["exp_avg"].data_ptr(),
                          st["exp_avg_sq"].data_ptr(), p.numel(), ctypes.c_float(group["lr"]), ctypes.c_float(b1),
                          ctypes.c_float(b2), ctypes.c_float(group["eps"]), st["step"], int(group["clamp"]),
                          None if mask is None else mask.data_ptr(), int(group["fixed_mode"]),
                          int(group["stride"]), torch.cuda.current_stream(p.device).cuda_stream)
        return loss


class _L2Loss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, target):
        image = image.contiguous()
        target = target.contiguous()
        n = image.numel()
        adj = torch.empty_like(image)
        loss = torch.zeros(1, dtype=torch.float32, device=image.device)
        _lib.call("dtv_loss_l2", image.data_ptr(), target.data_ptr(), n, ctypes.c_float(1.0 / n),
                  adj.data_ptr(), loss.data_ptr(), torch.cuda.current_stream(image.device).cuda_stream)
        ctx.save_for_backward(adj)
        return loss[0]

    @staticmethod
    def backward(ctx, grad_out):
        (adj,) = ctx.saved_tensors
        return adj * grad_out, None


def l2_loss(image: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """mean((image - target)^2); gradient 2 (image - target) / N."""
    return _L2Loss.apply(image, target)
