"""Renderer: the renderer object of the `difftetvr` module
(TetMeshVolumeRenderer, src/Renderer/TetMeshVolumeRenderer.hpp:84-280, bound in
src/Module/Module.cpp:838-981), backed by the CUDA library through the C ABI.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .tet_mesh import TetMesh
from .types import ColorStorage, RendererType, vec4


def linked_list_view(offsets: np.ndarray, records: np.ndarray, width: int, height: int):
    """(nodes u32[N, 3] = (bits, depth bits, next), heads i32[H, W]) from the
    offsets [P+1] / sorted records [N] layout; next and empty heads are -1."""
    off = np.asarray(offsets, np.int64)
    rec = np.asarray(records, np.uint64)
    n = rec.shape[0]
    nodes = np.empty((n, 3), np.uint32)
    nodes[:, 0] = (rec & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    nodes[:, 1] = (rec >> np.uint64(32)).astype(np.uint32)
    nxt = np.arange(1, n + 1, dtype=np.int64)
    ends = off[1:][np.diff(off) > 0] - 1  # last node of every non-empty list
    nxt[ends] = -1
    nodes[:, 2] = nxt.astype(np.int64).astype(np.uint32)
    counts = np.diff(off)
    heads = np.where(counts > 0, off[:-1], -1).astype(np.int32).reshape(height, width)
    return nodes, heads


def default_view_matrix() -> list[float]:
    """Camera at (0, 0, 0.8) with identity orientation (Module.cpp:458-463), column-major."""
    m = np.eye(4, dtype=np.float64)
    m[2, 3] = -0.8
    return [float(m[j, i]) for i in range(4) for j in range(4)]


class Renderer:
    STAGES = ("project", "count", "scan", "fill", "sort", "composite", "adjoint")

    def __init__(self, renderer_type: RendererType = RendererType.PPLL):
        renderer_type = RendererType(renderer_type)
        if renderer_type == RendererType.PROJECTION:
            raise RuntimeError(f"RendererType.{renderer_type.name} is not provided by difftetvr_b200")
        self._type = renderer_type
        h = ctypes.c_void_p()
        _lib.call("dtv_renderer_create", int(renderer_type), ctypes.byref(h))
        self._handle = h
        self._owner = True
        self._tet_mesh: TetMesh | None = None
        # Defaults of the reference (TetMeshVolumeRenderer.hpp:237-244, Module.cpp:458-463).
        self._attenuation = 100.0
        self._use_ert = True
        self._ert_thresh = 1e-4
        self._clear = (0.0, 0.0, 0.0, 0.0)
        self._width, self._height = 1, 1
        self._fovy = math.atan(1.0 / 2.0) * 2.0
        self._znear, self._zfar = 0.01, 100.0
        self._view = default_view_matrix()
        self._fragment_budget = 0
        self._over_budget = _lib.DTV_OVER_BUDGET_RECOMPUTE
        self._coarse_to_fine_target = 0
        self._export_lists = False
        self._last_image: torch.Tensor | None = None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if (h is not None and getattr(self, "_owner", False) and h.value and _lib is not None
                and getattr(_lib, "_lib", None) is not None):
            _lib.load().dtv_renderer_destroy(h)
            self._handle = None

    # -- settings (Module.cpp:862-911) -----------------------------------
    def get_renderer_type(self) -> RendererType:
        return self._type

    def set_tet_mesh(self, tet_mesh: TetMesh) -> None:
        self._tet_mesh = tet_mesh

    def get_tet_mesh(self) -> TetMesh:
        return self._tet_mesh

    def get_attenuation(self) -> float:
        return self._attenuation

    def set_attenuation(self, attenuation_coefficient: float) -> None:
        self._attenuation = float(attenuation_coefficient)

    def set_coarse_to_fine_target_num_tets(self, target_num_tets: int) -> None:
        self._coarse_to_fine_target = int(target_num_tets)

    def set_use_early_ray_termination(self, use_early_ray_termination: bool) -> None:
        self._use_ert = bool(use_early_ray_termination)

    def set_early_ray_out_thresh(self, threshold: float) -> None:
        self._ert_thresh = float(threshold)

    def set_early_ray_out_alpha(self, alpha: float) -> None:
        self._ert_thresh = 1.0 - float(alpha)

    def set_clear_color(self, color: vec4) -> None:
        self._clear = tuple(float(c) for c in color)

    def set_viewport_size(self, image_width: int, image_height: int, recreate_swapchain: bool = True) -> None:
        self._width, self._height = int(image_width), int(image_height)

    def get_viewport_size(self) -> tuple[int, int]:
        return self._width, self._height

    def reuse_intermediate_buffers_from(self, renderer_other: "Renderer") -> None:
        """Share the other renderer's fragment storage (Module.cpp:888-899)."""
        if self._owner and self._handle is not None and self._handle.value:
            _lib.load().dtv_renderer_destroy(self._handle)
        self._handle = renderer_other._handle
        self._owner = False
        self._keepalive = renderer_other

    def set_camera_fovy(self, fovy: float) -> None:
        self._fovy = float(fovy)

    def set_camera_clip(self, znear: float, zfar: float) -> None:
        self._znear, self._zfar = float(znear), float(zfar)

    def set_view_matrix(self, view_matrix_array) -> None:
        """16 floats, column-major (Module.cpp:904-911)."""
        arr = [float(v) for v in np.asarray(view_matrix_array, dtype=np.float64).reshape(-1)]
        if len(arr) != 16:
            raise RuntimeError("Error in set_view_matrix: expected 16 values.")
        self._view = arr

    def set_fragment_budget_bytes(self, budget: int, over_budget: str = "recompute") -> None:
        """Bound on the fragment records held at once (0 = none).  Over it,
        over_budget="recompute" renders in row bands that each fit and rebuilds
        each band's lists in render_adjoint (the lists are not stored);
        over_budget="error" raises RuntimeError (DTV_ERR_BUDGET)."""
        if over_budget not in ("recompute", "error"):
            raise ValueError("over_budget must be 'recompute' or 'error'")
        self._fragment_budget = int(budget)
        self._over_budget = _lib.DTV_OVER_BUDGET_RECOMPUTE if over_budget == "recompute" else \
            _lib.DTV_OVER_BUDGET_ERROR

    # -- kernel configuration (difftetvr_b200.autotune chooses it) -----------
    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        _lib.call("dtv_renderer_get_tuning", self._handle, ctypes.byref(t))
        return {"composite_tile": t.composite_tile, "adjoint_tile": t.adjoint_tile,
                "sort_surrogate_classes": t.sort_surrogate_classes, "sort_bucket_classes": t.sort_bucket_classes}

    def set_tuning(self, composite_tile: int | None = None, adjoint_tile: int | None = None,
                   sort_surrogate_classes: int | None = None, sort_bucket_classes: int | None = None) -> None:
        """Pixel tile of the composite blocks (0: 16x16, 1: 32x8, 2: 8x32) and
        of the adjoint blocks (0: 16x8, 1: 32x4, 2: 8x16), and the sort method per list-length class c = 1..4: depth
        buckets (bit c of sort_bucket_classes), else 32-bit surrogate keys (bit
        c of sort_surrogate_classes), else the 64-bit network.  Results are
        identical for every setting."""
        cur = self.get_tuning()
        pick = lambda v, k: cur[k] if v is None else int(v)
        t = _lib.Tuning(pick(composite_tile, "composite_tile"), pick(adjoint_tile, "adjoint_tile"),
                        pick(sort_surrogate_classes, "sort_surrogate_classes"),
                        pick(sort_bucket_classes, "sort_bucket_classes"))
        _lib.call("dtv_renderer_set_tuning", self._handle, ctypes.byref(t))

    def get_num_bands(self) -> int:
        """0 if the last render stored its fragment lists whole, else the number
        of row bands it ran in (each recomputed by render_adjoint)."""
        n = ctypes.c_int32()
        _lib.call("dtv_renderer_get_num_bands", self._handle, ctypes.byref(n))
        return int(n.value)

    # -- render / adjoint (Module.cpp:912-959) ----------------------------
    def _camera(self) -> _lib.Camera:
        cam = _lib.Camera()
        cam.view[:] = self._view
        cam.fovy = self._fovy
        cam.znear = self._znear
        cam.zfar = self._zfar
        cam.width = self._width
        cam.height = self._height
        return cam

    def _params(self, use_abs_grad: bool = False) -> _lib.RenderParams:
        p = _lib.RenderParams()
        p.attenuation = self._attenuation
        # Early ray termination only when gradients are on, as in the reference
        # (USE_TERMINATION_INDEX, TetMeshVolumeRenderer.cpp:417-419).
        mesh = self._tet_mesh
        p.use_early_ray_termination = int(self._use_ert and mesh is not None and mesh._use_gradients)
        p.early_ray_out_thresh = self._ert_thresh
        p.clear_color[:] = self._clear
        p.use_abs_grad = int(use_abs_grad)
        p.fragment_budget_bytes = self._fragment_budget
        p.over_budget = self._over_budget
        return p

    def render(self) -> torch.Tensor:
        mesh = self._tet_mesh
        if mesh is None or mesh.get_is_empty():
            raise RuntimeError("Missing valid tet mesh in Renderer.render.")
        pos = mesh.get_vertex_positions().detach()
        cells = mesh.get_color_storage() == ColorStorage.PER_CELL
        col = (mesh.get_cell_colors() if cells else mesh.get_vertex_colors()).detach()
        image = torch.empty((self._height, self._width, 4), dtype=torch.float32, device=pos.device)
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        cam, prm = self._camera(), self._params()
        _lib.call("dtv_renderer_render_cells" if cells else "dtv_renderer_render", self._handle,
                  mesh.native.handle, pos.data_ptr(), col.data_ptr(), ctypes.byref(cam), ctypes.byref(prm),
                  image.data_ptr(), stream)
        self._last_image = image
        return image

    def _check_adjoint(self, image_adjoint: torch.Tensor, name: str):
        mesh = self._tet_mesh
        if mesh is None or mesh.get_is_empty():
            raise RuntimeError(f"Missing valid tet mesh in Renderer.{name}.")
        pos = mesh.get_vertex_positions()
        if not torch.is_tensor(image_adjoint) or image_adjoint.device != pos.device:
            raise RuntimeError(
                "Error in render_adjoint: The tensors must be on the device used at initialization time.")
        if image_adjoint.dim() != 3:
            raise RuntimeError("Error in render_adjoint: imageAdjointTensor.sizes().size() != 3.")
        if image_adjoint.shape[2] != 4:
            raise RuntimeError("Error in render_adjoint: The number of image channels is not equal to 4.")
        if image_adjoint.dtype != torch.float32:
            raise RuntimeError("Error in render_adjoint: The only data type currently supported is 32-bit float.")
        if tuple(image_adjoint.shape[:2]) != (self._height, self._width):
            raise RuntimeError("Error in render_adjoint: image size does not match the viewport.")
        return mesh, image_adjoint.contiguous()

    def _adjoint(self, mesh: TetMesh, image_adjoint: torch.Tensor, use_abs_grad: bool, grad_positions: torch.Tensor,
                 grad_colors: torch.Tensor) -> None:
        """grad_colors: [V, 4] per-vertex or [T, 4] per-cell, by the mesh's colour storage."""
        pos = mesh.get_vertex_positions()
        cells = mesh.get_color_storage() == ColorStorage.PER_CELL
        col = mesh.get_cell_colors() if cells else mesh.get_vertex_colors()
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        _lib.call("dtv_renderer_render_adjoint_cells" if cells else "dtv_renderer_render_adjoint", self._handle,
                  mesh.native.handle, pos.detach().data_ptr(), col.detach().data_ptr(), image_adjoint.data_ptr(),
                  int(bool(use_abs_grad)), grad_positions.data_ptr(), grad_colors.data_ptr(), stream)

    def render_adjoint(self, image_adjoint: torch.Tensor, use_abs_grad: bool = False) -> None:
        """Adds the vertex position / colour gradients into the mesh tensors' .grad
        (Module.cpp:922-959)."""
        mesh, image_adjoint = self._check_adjoint(image_adjoint, "render_adjoint")
        pos = mesh.get_vertex_positions()
        col = mesh.get_cell_colors() if mesh.get_color_storage() == ColorStorage.PER_CELL else \
            mesh.get_vertex_colors()
        if pos.grad is None:
            pos.grad = torch.zeros_like(pos)
        if col.grad is None:
            col.grad = torch.zeros_like(col)
        self._adjoint(mesh, image_adjoint, use_abs_grad, pos.grad, col.grad)

    def render_adjoint_into(self, image_adjoint: torch.Tensor, grad_positions: torch.Tensor,
                            grad_colors: torch.Tensor, use_abs_grad: bool = False) -> None:
        """Adds the gradients into caller-owned contiguous float32 tensors
        [V, 3] / [V, 4] (grad_colors 16-byte aligned) instead of .grad."""
        mesh, image_adjoint = self._check_adjoint(image_adjoint, "render_adjoint_into")
        V = mesh.get_num_vertices()
        Nc = mesh.get_num_cells() if mesh.get_color_storage() == ColorStorage.PER_CELL else V
        for t, rows, c in ((grad_positions, V, 3), (grad_colors, Nc, 4)):
            if (not torch.is_tensor(t) or t.dtype != torch.float32 or not t.is_contiguous()
                    or tuple(t.shape) != (rows, c) or t.device != image_adjoint.device):
                raise RuntimeError(f"Error in render_adjoint_into: gradient tensors must be contiguous float32 "
                                   f"[{V}, 3] / [{Nc}, 4] on the mesh's device.")
        self._adjoint(mesh, image_adjoint, use_abs_grad, grad_positions, grad_colors)

    # -- fragment list export (Module.cpp:960-981) -------------------------
    def set_export_linked_list_data(self) -> None:
        self._export_lists = True

    def get_num_fragments(self) -> int:
        n = ctypes.c_uint64()
        _lib.call("dtv_renderer_get_num_fragments", self._handle, ctypes.byref(n))
        return int(n.value)

    def get_fragment_lists(self) -> tuple[np.ndarray, np.ndarray]:
        """(offsets u64[H*W+1], records u64[Nf]) of the last render, sorted per pixel."""
        nf = self.get_num_fragments()
        offsets = np.empty(self._width * self._height + 1, dtype=np.uint64)
        records = np.empty(max(nf, 1), dtype=np.uint64)
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("dtv_renderer_copy_fragments", self._handle, offsets.ctypes.data, records.ctypes.data,
                  records.shape[0], stream)
        return offsets, records[:nf]

    def get_fragment_buffer(self) -> torch.Tensor:
        """Sorted fragment records as int64 [Nf]:
        (fp32 view-depth bits << 32) | (faceIndex << 2) | (boundary << 1) | frontFacing."""
        _, rec = self.get_fragment_lists()
        return torch.from_numpy(rec.view(np.int64).copy())

    def get_start_offset_buffer(self) -> torch.Tensor:
        """Per-pixel list offsets as int64 [H*W+1] (pixel p owns records [o[p], o[p+1]))."""
        off, _ = self.get_fragment_lists()
        return torch.from_numpy(off.view(np.int64).copy())

    def get_linked_list_buffers(self) -> tuple[torch.Tensor, torch.Tensor]:
        """The fragment lists in the layout of the reference's PPLL export
        (get_fragment_buffer [N, 3] float32 / get_start_offset_buffer [H, W]
        int32, TetMeshRendererPPLL.cpp:816-860): node i = (bits, depth, next)
        with the uint fields stored as float32 bit patterns, bits = face << 2 |
        boundary << 1 | front, next = index of the next node or -1 (0xFFFFFFFF),
        head = -1 for empty pixels.  Here the lists are in front-to-back order
        and the depth is view depth (the reference stores NDC depth)."""
        off, rec = self.get_fragment_lists()
        nodes, heads = linked_list_view(off, rec, self._width, self._height)
        return torch.from_numpy(nodes.view(np.float32)), torch.from_numpy(heads)

    def get_pixel_state(self) -> tuple[np.ndarray, np.ndarray]:
        """(final transmittance f32[H,W], termination index u32[H,W]) of the last render."""
        t = np.empty(self._width * self._height, dtype=np.float32)
        term = np.empty(self._width * self._height, dtype=np.uint32)
        _lib.call("dtv_renderer_copy_pixel_state", self._handle, t.ctypes.data, term.ctypes.data,
                  torch.cuda.current_stream().cuda_stream)
        return t.reshape(self._height, self._width), term.reshape(self._height, self._width)

    # -- tracing -----------------------------------------------------------
    def set_stage_timing(self, enable: bool = True) -> None:
        _lib.call("dtv_renderer_set_timing", self._handle, int(bool(enable)))

    def get_stage_times(self) -> dict[str, float]:
        ms = (ctypes.c_float * len(self.STAGES))()
        _lib.call("dtv_renderer_stage_times", self._handle, ms, len(self.STAGES))
        return {k: float(v) for k, v in zip(self.STAGES, ms)}
