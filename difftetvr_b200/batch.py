"""Batched multi-view / multi-mesh rendering, adjoint and training steps.

``BatchRenderer`` drives the C ABI's ``dtv_batch_*`` entry points: many
camera views of several meshes (of uneven size and resolution) go through the
hot path with one kernel launch per stage, and a whole training step
(render, L2 loss, adjoint, Adam of every mesh) can be captured once as a CUDA
graph and replayed.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import torch

from . import _lib
from .tet_mesh import TetMesh


@dataclass
class View:
    """One view of a batch: mesh index, camera and viewport."""

    mesh: int
    view_matrix: list
    width: int
    height: int
    fovy: float = math.radians(45.0)
    znear: float = 0.01
    zfar: float = 100.0
    target: torch.Tensor | None = None           # train_step: target image [H, W, 4]
    image_adjoint: torch.Tensor | None = None    # render_adjoint: dL/dimage [H, W, 4]
    grad_slot: int = -1                          # render_adjoint: gradient slot index
    image: torch.Tensor | None = field(default=None, repr=False)  # output buffer (allocated if None)


class BatchRenderer:
    """Renders and differentiates batches of views of the given meshes."""

    def __init__(self, meshes: list[TetMesh], attenuation: float = 1.0, use_early_ray_termination: bool = True,
                 early_ray_out_thresh: float = 1e-4, clear_color=(0.0, 0.0, 0.0, 0.0)):
        h = ctypes.c_void_p()
        _lib.call("dtv_batch_create", ctypes.byref(h))
        self._handle = h
        self.attenuation = float(attenuation)
        self.use_ert = bool(use_early_ray_termination)
        self.ert_thresh = float(early_ray_out_thresh)
        self.clear = tuple(float(c) for c in clear_color)
        self.set_meshes(meshes)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value and _lib is not None and getattr(_lib, "_lib", None) is not None:
            _lib.load().dtv_batch_destroy(h)
            self._handle = None

    def set_meshes(self, meshes: list[TetMesh]) -> None:
        from .types import ColorStorage
        if any(m.get_color_storage() != ColorStorage.PER_VERTEX for m in meshes):
            raise RuntimeError("BatchRenderer renders ColorStorage.PER_VERTEX meshes; use Renderer for PER_CELL.")
        self.meshes = list(meshes)
        n = len(self.meshes)
        arr_m = (ctypes.c_void_p * n)(*[m.native.handle.value for m in self.meshes])
        arr_p = (ctypes.c_void_p * n)(*[m.get_vertex_positions().data_ptr() for m in self.meshes])
        arr_c = (ctypes.c_void_p * n)(*[m.get_vertex_colors().data_ptr() for m in self.meshes])
        _lib.call("dtv_batch_set_meshes", self._handle, n, arr_m, arr_p, arr_c)

    def reserve(self, max_views: int, max_vertices: int, max_pixels: int, max_fragments: int,
                max_grad_vertices: int) -> None:
        """Allocates scratch for batches up to these sizes now (dtv_batch_reserve),
        so serving never allocates device memory between batches."""
        import torch
        _lib.call("dtv_batch_reserve", self._handle, int(max_views), int(max_vertices), int(max_pixels),
                  int(max_fragments), int(max_grad_vertices), torch.cuda.current_stream().cuda_stream)

    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        _lib.call("dtv_batch_get_tuning", self._handle, ctypes.byref(t))
        return {"sort_surrogate_classes": t.sort_surrogate_classes, "sort_bucket_classes": t.sort_bucket_classes}

    def set_tuning(self, sort_surrogate_classes: int | None = None, sort_bucket_classes: int | None = None) -> None:
        """Sort method per list-length class c = 1..4: depth buckets (bit c
        of sort_bucket_classes), else 32-bit surrogate keys (bit c of
        sort_surrogate_classes), else the 64-bit network; identical results."""
        cur = self.get_tuning()
        t = _lib.Tuning(0, 0, cur["sort_surrogate_classes"] if sort_surrogate_classes is None
                        else int(sort_surrogate_classes),
                        cur["sort_bucket_classes"] if sort_bucket_classes is None else int(sort_bucket_classes))
        _lib.call("dtv_batch_set_tuning", self._handle, ctypes.byref(t))

    def set_graph(self, enable: bool = True) -> None:
        _lib.call("dtv_batch_set_graph", self._handle, int(bool(enable)))

    def info(self) -> dict:
        nf, cap, rerun = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        g = ctypes.c_int32()
        _lib.call("dtv_batch_get_info", self._handle, ctypes.byref(nf), ctypes.byref(cap), ctypes.byref(rerun),
                  ctypes.byref(g))
        return {"fragments": nf.value, "capacity": cap.value, "steps_rerun": rerun.value, "graph": bool(g.value)}

    # -- helpers -------------------------------------------------------------
    def _params(self) -> _lib.RenderParams:
        p = _lib.RenderParams()
        p.attenuation = self.attenuation
        p.use_early_ray_termination = int(self.use_ert)
        p.early_ray_out_thresh = self.ert_thresh
        p.clear_color[:] = self.clear
        return p

    def _views(self, views: list[View], device) -> ctypes.Array:
        arr = (_lib.BatchView * len(views))()
        for i, v in enumerate(views):
            if v.image is None or tuple(v.image.shape) != (v.height, v.width, 4):
                v.image = torch.empty((v.height, v.width, 4), dtype=torch.float32, device=device)
            b = arr[i]
            b.mesh = int(v.mesh)
            b.grad_slot = int(v.grad_slot)
            b.camera.view[:] = [float(x) for x in v.view_matrix]
            b.camera.fovy = float(v.fovy)
            b.camera.znear, b.camera.zfar = float(v.znear), float(v.zfar)
            b.camera.width, b.camera.height = int(v.width), int(v.height)
            b.d_image = v.image.data_ptr()
            b.d_target = v.target.contiguous().data_ptr() if v.target is not None else None
            b.d_image_adjoint = v.image_adjoint.contiguous().data_ptr() if v.image_adjoint is not None else None
        return arr

    # -- entry points ----------------------------------------------------------
    def render(self, views: list[View]) -> list[torch.Tensor]:
        device = self.meshes[0].get_vertex_positions().device
        arr = self._views(views, device)
        prm = self._params()
        _lib.call("dtv_batch_render", self._handle, len(views), arr, ctypes.byref(prm),
                  torch.cuda.current_stream(device).cuda_stream)
        self._last_views = views
        return [v.image for v in views]

    def render_async(self, views: list[View]) -> list[torch.Tensor]:
        """render() without a host synchronisation, bounded by the reserved
        record capacity (reserve()); check render_status() once the stream has
        passed it and call render() again if it did not fit."""
        device = self.meshes[0].get_vertex_positions().device
        arr = self._views(views, device)
        prm = self._params()
        _lib.call("dtv_batch_render_async", self._handle, len(views), arr, ctypes.byref(prm),
                  torch.cuda.current_stream(device).cuda_stream)
        self._last_views = views
        return [v.image for v in views]

    def render_status(self) -> tuple[bool, int]:
        """(fit, fragments) of the last render_async (its stream must be past it)."""
        fits, nf = ctypes.c_int32(), ctypes.c_uint64()
        _lib.call("dtv_batch_render_status", self._handle, ctypes.byref(fits), ctypes.byref(nf))
        return bool(fits.value), int(nf.value)

    def render_adjoint(self, slots: list[tuple[int, torch.Tensor, torch.Tensor]], use_abs_grad: bool = False):
        """slots: (mesh index, grad_positions [V,3], grad_colors [V,4]) per gradient slot;
        views of the last render() name their slot in View.grad_slot."""
        arr = (_lib.BatchGradSlot * max(len(slots), 1))()
        for i, (m, gp, gc) in enumerate(slots):
            arr[i].mesh = int(m)
            arr[i].d_grad_positions = gp.data_ptr()
            arr[i].d_grad_colors = gc.data_ptr()
        device = self.meshes[0].get_vertex_positions().device
        views = self._last_views
        varr = self._views(views, device)
        _lib.call("dtv_batch_render_adjoint", self._handle, len(views), varr, len(slots), arr,
                  int(bool(use_abs_grad)), torch.cuda.current_stream(device).cuda_stream)

    def train_step(self, views: list[View], lr_positions: float = 1e-4, lr_colors: float = 1e-2,
                   betas=(0.9, 0.999), eps: float = 1e-8, clamp_colors: int = 1,
                   fixed_boundary: int = 0) -> torch.Tensor:
        """Render all views, L2 loss against each view's target (mean per view,
        summed), adjoint, and an Adam step of every mesh's positions and colours
        (in place).  Returns the loss as a 0-d CUDA tensor."""
        device = self.meshes[0].get_vertex_positions().device
        arr = self._views(views, device)
        prm = self._params()
        opt = _lib.BatchOptim()
        opt.lr_positions, opt.lr_colors = float(lr_positions), float(lr_colors)
        opt.beta1, opt.beta2, opt.eps = float(betas[0]), float(betas[1]), float(eps)
        opt.clamp_colors, opt.fixed_boundary = int(clamp_colors), int(fixed_boundary)
        loss = torch.zeros(1, dtype=torch.float32, device=device)
        _lib.call("dtv_batch_train_step", self._handle, len(views), arr, ctypes.byref(prm), ctypes.byref(opt),
                  loss.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
        return loss[0]
