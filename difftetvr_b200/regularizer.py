"""TetRegularizer: the reference's difftetvr.TetRegularizer (Module.cpp:663-695,
983-995), penalising badly shaped (and inverted) tets through a mirrored
softplus of the Parthasarathy quality measure; compute_grad() ADDS the
gradient into the mesh's vertex-position .grad, as the reference adds into its
gradient buffer before Renderer.render_adjoint (pytests/pyutils.py:45-46)."""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .tet_mesh import TetMesh


class TetRegularizer:
    def __init__(self, tet_mesh: TetMesh, reg_lambda: float, softplus_beta: float):
        if softplus_beta <= 0:
            raise RuntimeError("TetRegularizer: softplus_beta must be > 0.")
        self.tet_mesh = tet_mesh
        self.reg_lambda = float(reg_lambda)
        self.softplus_beta = float(softplus_beta)

    def _run(self, grad: torch.Tensor, loss: torch.Tensor | None) -> None:
        pos = self.tet_mesh.get_vertex_positions()
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        _lib.call("dtv_tet_regularizer_grad", self.tet_mesh.native.handle, pos.detach().data_ptr(),
                  ctypes.c_float(self.reg_lambda), ctypes.c_float(self.softplus_beta), grad.data_ptr(),
                  None if loss is None else loss.data_ptr(), stream)

    def compute_grad(self) -> None:
        """Adds d(penalty)/d(positions) into the vertex positions' .grad."""
        pos = self.tet_mesh.get_vertex_positions()
        if pos.grad is None:
            pos.grad = torch.zeros_like(pos)
        self._run(pos.grad, None)

    def compute_grad_into(self, grad_positions: torch.Tensor) -> torch.Tensor:
        """Adds the gradient into a caller-owned contiguous float32 [V, 3]
        tensor and returns the penalty summed over tets (a 1-element tensor)."""
        V = self.tet_mesh.get_num_vertices()
        if (grad_positions.dtype != torch.float32 or not grad_positions.is_contiguous()
                or tuple(grad_positions.shape) != (V, 3)):
            raise RuntimeError(f"TetRegularizer: gradient tensor must be contiguous float32 [{V}, 3].")
        loss = torch.zeros(1, dtype=torch.float32, device=grad_positions.device)
        self._run(grad_positions, loss)
        return loss
