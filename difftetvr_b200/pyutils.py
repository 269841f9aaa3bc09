"""Autograd wrappers (pytests/pyutils.py:31-79 of the reference).

``DifferentiableRenderingFunction`` keeps the reference signature for drop-in
use: forward renders, backward calls ``render_adjoint`` which ADDS the vertex
position / colour gradients into the tensors' ``.grad`` in place and returns
None for every input.  ``RenderFunction`` is the pure form that returns the
gradients explicitly (used by batching and serving).
"""
from __future__ import annotations

import torch

from .types import ColorStorage


class DifferentiableRenderingFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer, tet_regularizer, use_abs_grad, vertex_positions, colors):
        image = renderer.render()
        ctx.save_for_backward(image)
        ctx.renderer = renderer
        ctx.tet_regularizer = tet_regularizer
        ctx.use_abs_grad = use_abs_grad
        return image

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, image_adj):
        if ctx.tet_regularizer is not None:
            ctx.tet_regularizer.compute_grad()
        ctx.renderer.render_adjoint(image_adj, ctx.use_abs_grad)
        del ctx.renderer
        del ctx.tet_regularizer
        del ctx.use_abs_grad
        return None, None, None, None, None


class DifferentiableRenderer(torch.nn.Module):
    def __init__(self, renderer, use_tet_regularizer: bool = False, tet_reg_lambda: float = 0.0,
                 tet_reg_softplus_beta: float = 1.0):
        super().__init__()
        self.renderer = renderer
        self.use_abs_grad = False
        self.tet_regularizer = None
        if use_tet_regularizer:
            from .regularizer import TetRegularizer
            self.tet_regularizer = TetRegularizer(renderer.get_tet_mesh(), tet_reg_lambda, tet_reg_softplus_beta)

    def set_use_abs_grad(self, use_abs_grad):
        self.use_abs_grad = use_abs_grad

    def forward(self):
        tet_mesh = self.renderer.get_tet_mesh()
        vertex_positions = tet_mesh.get_vertex_positions()
        if tet_mesh.get_color_storage() == ColorStorage.PER_VERTEX:
            colors = tet_mesh.get_vertex_colors()
        else:
            colors = tet_mesh.get_cell_colors()
        return DifferentiableRenderingFunction.apply(
            self.renderer, self.tet_regularizer, self.use_abs_grad, vertex_positions, colors)


class RenderFunction(torch.autograd.Function):
    """image = RenderFunction.apply(renderer, positions, colors); backward returns
    (None, d_positions, d_colors) as fresh tensors (the mesh's .grad is untouched)."""

    @staticmethod
    def forward(ctx, renderer, positions, colors):
        image = renderer.render()
        ctx.renderer = renderer
        ctx.save_for_backward(positions, colors)
        return image

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, image_adj):
        positions, colors = ctx.saved_tensors
        gp = torch.zeros_like(positions)
        gc = torch.zeros_like(colors)
        ctx.renderer.render_adjoint_into(image_adj.contiguous(), gp, gc)
        return None, gp, gc
