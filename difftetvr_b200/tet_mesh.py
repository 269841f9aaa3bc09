"""TetMesh: the mesh object of the `difftetvr` module (src/Tet/TetMesh.hpp:89-286,
bound in src/Module/Module.cpp:775-837), holding cells, per-vertex positions
and RGBA as CUDA tensors and the face topology on the device.

As in the reference, ``get_vertex_positions()`` / ``get_vertex_colors()``
return the same leaf tensors every call, with ``.grad`` attached; the renderer
adds gradients into those ``.grad`` buffers in place (TetMesh.cpp:236-308), so
``torch.optim`` updates the tensors the renderer reads.  Gradient buffers start
at zero (the reference fills them with a copy of the values,
TetMesh.cpp:661-675; callers zero them before use either way).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .types import AABB3, ColorStorage, SplitGradientType, TestCase, vec3, vec4

# HEX_TO_TET_TABLE, src/Tet/TetMesh.cpp:104-117 (Kuhn split around diagonal 0-6).
HEX_TO_TET_TABLE = np.array([[0, 4, 7, 6], [0, 4, 6, 5], [0, 3, 6, 7], [0, 3, 2, 6], [0, 1, 5, 6], [0, 1, 6, 2]],
                            dtype=np.int64)


def convert_hex_to_tet_indices(hex_indices: np.ndarray) -> np.ndarray:
    """convertHexToTetIndices (TetMesh.cpp:119-132): 8 vertex ids per hex -> 6 tets."""
    hexes = np.asarray(hex_indices, dtype=np.uint32).reshape(-1, 8)
    return hexes[:, HEX_TO_TET_TABLE].reshape(-1, 4).astype(np.uint32)


def build_hex_mesh(aabb_min, aabb_max, xs: int, ys: int, zs: int):
    """Vertex grid and Kuhn tets of TetMesh::setHexMeshConst (C ABI dtv_build_hex_mesh).

    Returns (cells u32[T,4], positions f32[V,3]) on the host."""
    nv = xs * ys * zs
    nt = 6 * (xs - 1) * (ys - 1) * (zs - 1)
    cells = np.empty((nt, 4), dtype=np.uint32)
    pos = np.empty((nv, 3), dtype=np.float32)
    mn = (ctypes.c_float * 3)(*aabb_min)
    mx = (ctypes.c_float * 3)(*aabb_max)
    _lib.call("dtv_build_hex_mesh", mn, mx, xs, ys, zs, cells.ctypes.data, pos.ctypes.data)
    return cells, pos


def build_faces_host(cells: np.ndarray, num_vertices: int):
    """Unique faces (C ABI dtv_mesh_build_faces_host; buildFacesSlim, TetMesh.cpp:1218-1268).

    Returns (tri u32[F,3], face_boundary u32[F], face_to_tet u32[F,2], vertex_boundary u32[V])."""
    cells = np.ascontiguousarray(cells, dtype=np.uint32).reshape(-1, 4)
    T = cells.shape[0]
    tri = np.empty((4 * T, 3), dtype=np.uint32)
    fb = np.empty(4 * T, dtype=np.uint32)
    f2t = np.empty((4 * T, 2), dtype=np.uint32)
    vb = np.empty(num_vertices, dtype=np.uint32)
    nf = ctypes.c_uint64(0)
    _lib.call("dtv_mesh_build_faces_host", cells.ctypes.data, T, num_vertices, tri.ctypes.data, fb.ctypes.data,
              f2t.ctypes.data, vb.ctypes.data, ctypes.byref(nf))
    F = nf.value
    return tri[:F].copy(), fb[:F].copy(), f2t[:F].copy(), vb


def unlink_cells(cells: np.ndarray, positions: np.ndarray, vertex_colors: np.ndarray | None = None):
    """TetMesh::unlinkTets (TetMesh.cpp:1950-1989) on host arrays: every cell
    gets its own four vertices (vertex 4 t + k is corner k of cell t), so no
    face is shared any more.

    Returns (cells u32[T,4], positions f32[4T,3], vertex colours f32[4T,4] or None)."""
    flat = np.asarray(cells, dtype=np.uint32).reshape(-1)
    new_cells = np.arange(flat.size, dtype=np.uint32).reshape(-1, 4)
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32)[flat])
    col = None if vertex_colors is None else np.ascontiguousarray(np.asarray(vertex_colors, dtype=np.float32)[flat])
    return new_cells, pos, col


def remove_transparent_cells(cells: np.ndarray, positions: np.ndarray, vertex_colors: np.ndarray | None,
                             cell_colors: np.ndarray | None, alpha_threshold: float):
    """TetMesh::removeTransparentTets (TetMesh.cpp:1991-2084) on host arrays.

    A cell stays when one of its vertices has alpha >= alpha_threshold
    (per-vertex colours) or its own alpha is >= alpha_threshold (per-cell
    colours).  The vertices the kept cells use stay, in their original order,
    and the kept cells keep their order.

    Returns (cells u32[T',4], positions f32[V',3], vertex colours or None,
    cell colours or None)."""
    cells = np.asarray(cells, dtype=np.uint32).reshape(-1, 4)
    pos = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    thr = np.float32(alpha_threshold)
    if vertex_colors is not None:
        vcol = np.asarray(vertex_colors, dtype=np.float32).reshape(-1, 4)
        keep = (vcol[cells, 3] >= thr).any(axis=1)
    else:
        ccol = np.asarray(cell_colors, dtype=np.float32).reshape(-1, 4)
        keep = ccol[:, 3] >= thr
    kept = cells[keep]
    used = np.zeros(pos.shape[0], dtype=bool)
    used[kept.reshape(-1)] = True
    new_index = (np.cumsum(used) - used).astype(np.uint32)  # rank among the used vertices
    new_cells = np.ascontiguousarray(new_index[kept])
    new_pos = np.ascontiguousarray(pos[used])
    new_vcol = None if vertex_colors is None else np.ascontiguousarray(vcol[used])
    new_ccol = None if vertex_colors is not None else np.ascontiguousarray(ccol[keep])
    return new_cells, new_pos, new_vcol, new_ccol


class NativeMesh:
    """Owner of a dtv_mesh handle (device face topology)."""

    def __init__(self, cells: np.ndarray, num_vertices: int):
        cells = np.ascontiguousarray(cells, dtype=np.uint32).reshape(-1, 4)
        h = ctypes.c_void_p()
        _lib.call("dtv_mesh_create", cells.ctypes.data, cells.shape[0], num_vertices, ctypes.byref(h))
        self.handle = h
        nc, nv, nf = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _lib.call("dtv_mesh_get_info", h, ctypes.byref(nc), ctypes.byref(nv), ctypes.byref(nf))
        self.num_cells, self.num_vertices, self.num_faces = nc.value, nv.value, nf.value

    def copy_faces(self):
        F, V = self.num_faces, self.num_vertices
        tri = np.empty((F, 3), dtype=np.uint32)
        fb = np.empty(F, dtype=np.uint32)
        f2t = np.empty((F, 2), dtype=np.uint32)
        vb = np.empty(V, dtype=np.uint32)
        _lib.call("dtv_mesh_copy_faces", self.handle, tri.ctypes.data, fb.ctypes.data, f2t.ctypes.data,
                  vb.ctypes.data)
        return tri, fb, f2t, vb

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None and getattr(_lib, "_lib", None) is not None:
            _lib.load().dtv_mesh_destroy(h)
            self.handle = None


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("difftetvr_b200 runs on CUDA devices only (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


class TetMesh:
    """Tetrahedral mesh with per-vertex RGBA (A = extinction density)."""

    def __init__(self):
        self._cells: np.ndarray | None = None
        self._positions: torch.Tensor | None = None
        self._colors: torch.Tensor | None = None
        self._cell_colors: torch.Tensor | None = None
        self._use_gradients = False
        self._color_storage = ColorStorage.PER_VERTEX
        self._native: NativeMesh | None = None
        self._vertex_boundary: torch.Tensor | None = None
        self._force_ovm = False

    # -- construction ------------------------------------------------------
    def set_use_gradients(self, use_gradients: bool = True) -> None:
        """TetMesh::setUseGradients (Module.cpp:785)."""
        self._use_gradients = bool(use_gradients)
        if self._positions is not None:
            self._attach_grads()

    def set_tet_mesh_data(self, cells, vertex_positions, vertex_colors) -> None:
        """TetMesh::setTetMeshData(cells, positions, colors) (TetMesh.hpp:93-95)."""
        cells = np.ascontiguousarray(np.asarray(cells, dtype=np.uint32).reshape(-1, 4))
        pos = torch.as_tensor(np.asarray(vertex_positions, dtype=np.float32).reshape(-1, 3))
        col = torch.as_tensor(np.asarray(vertex_colors, dtype=np.float32).reshape(-1, 4))
        if col.shape[0] != pos.shape[0]:
            raise RuntimeError("Error in TetMesh.set_tet_mesh_data: #colors != #vertices.")
        if cells.size and int(cells.max()) >= pos.shape[0]:
            raise RuntimeError("Error in TetMesh.set_tet_mesh_data: cell index out of range.")
        dev = _device()
        self._cells = cells
        self._color_storage = ColorStorage.PER_VERTEX
        self._positions = pos.to(dev).contiguous()
        self._colors = col.to(dev).contiguous()
        self._cell_colors = None
        self._native = NativeMesh(cells, pos.shape[0])
        _, _, _, vb = self._native.copy_faces()
        self._vertex_boundary = torch.as_tensor(vb.astype(np.int32)).to(dev)
        self._attach_grads()

    def set_tet_mesh_data_cell(self, cells, vertex_positions, cell_colors) -> None:
        """TetMesh::setTetMeshDataCell: one RGBA per cell (ColorStorage.PER_CELL)."""
        cells = np.ascontiguousarray(np.asarray(cells, dtype=np.uint32).reshape(-1, 4))
        pos = torch.as_tensor(np.asarray(vertex_positions, dtype=np.float32).reshape(-1, 3))
        ccol = torch.as_tensor(np.asarray(cell_colors, dtype=np.float32).reshape(-1, 4))
        if ccol.shape[0] != cells.shape[0]:
            raise RuntimeError("Error in TetMesh.set_tet_mesh_data_cell: #colors != #cells.")
        if cells.size and int(cells.max()) >= pos.shape[0]:
            raise RuntimeError("Error in TetMesh.set_tet_mesh_data_cell: cell index out of range.")
        dev = _device()
        self._cells = cells
        self._color_storage = ColorStorage.PER_CELL
        self._positions = pos.to(dev).contiguous()
        self._colors = None
        self._cell_colors = ccol.to(dev).contiguous()
        self._native = NativeMesh(cells, pos.shape[0])
        _, _, _, vb = self._native.copy_faces()
        self._vertex_boundary = torch.as_tensor(vb.astype(np.int32)).to(dev)
        self._attach_grads()

    def _attach_grads(self) -> None:
        for t in (self._positions, self._colors, self._cell_colors):
            if t is None:
                continue
            t.requires_grad_(self._use_gradients)
            if self._use_gradients:
                if t.grad is None:
                    t.grad = torch.zeros_like(t)
            else:
                t.grad = None

    def load_test_data(self, test_case: TestCase) -> None:
        """TetMesh::loadTestData (TetMesh.cpp:1016-1077)."""
        if test_case == TestCase.SINGLE_TETRAHEDRON:
            cells = np.array([[0, 1, 2, 3]], dtype=np.uint32)
            pos = np.array([[-0.1, -0.1, 0.1], [0.1, -0.1, 0.1], [0.0, 0.3, 0.0], [0.1, -0.1, -0.1]],
                           dtype=np.float32)
            col = np.array([[1.0, 1.0, 1.0, 0.1], [1.0, 1.0, 1.0, 0.1], [0.0, 1.0, 0.0, 0.1],
                            [1.0, 1.0, 1.0, 0.8]], dtype=np.float32)
            self.set_tet_mesh_data(cells, pos, col)
        elif test_case == TestCase.CUBE_CENTRAL_GRADIENT:
            cells, pos, col = cube_central_gradient_data()
            self.set_tet_mesh_data(cells, pos, col)
        else:
            raise RuntimeError(f"Unknown test case {test_case}")

    def set_hex_mesh_const(self, aabb: AABB3, xs: int, ys: int, zs: int, const_color: vec4,
                           color_storage: ColorStorage = ColorStorage.PER_VERTEX) -> None:
        """TetMesh::setHexMeshConst (TetMesh.cpp:1882-1936); xs, ys, zs are vertex counts."""
        cells, pos = build_hex_mesh(tuple(aabb.min), tuple(aabb.max), xs, ys, zs)
        c = np.array(tuple(const_color), dtype=np.float32)
        if ColorStorage(color_storage) == ColorStorage.PER_CELL:
            self.set_tet_mesh_data_cell(cells, pos, np.tile(c, (cells.shape[0], 1)))
        else:
            self.set_tet_mesh_data(cells, pos, np.tile(c, (pos.shape[0], 1)))

    # -- coarse to fine (Module.cpp:820-832) ----------------------------------
    def split_by_largest_gradient_magnitudes(self, volume_renderer, split_gradient_type: SplitGradientType,
                                             splits_ratio: float) -> None:
        """TetMesh::splitByLargestGradientMagnitudes (TetMesh.cpp:1786-1881):
        the ceil(splits_ratio * V) vertices with the largest gradient magnitude
        (|d position| for POSITION / ABS_POSITION and for per-cell meshes,
        |d colour| otherwise) are subdivided in descending order, then the
        renderer is given the refined mesh.  Gradients are read from .grad."""
        V = self.get_num_vertices()
        gtype = SplitGradientType(split_gradient_type)
        use_pos = gtype in (SplitGradientType.POSITION, SplitGradientType.ABS_POSITION) or \
            self._color_storage == ColorStorage.PER_CELL
        g = (self._positions if use_pos else self._colors).grad
        mag = np.zeros(V, np.float32) if g is None else g.detach().norm(dim=1).float().cpu().numpy()
        num = min(int(np.ceil(float(splits_ratio) * V)), V)
        # Descending (magnitude, index) pairs, as a reverse sort of the pairs.
        order = np.lexsort((-np.arange(V), -mag.astype(np.float64)))[:num].astype(np.uint32)
        cells = np.ascontiguousarray(self._cells)
        pos = np.ascontiguousarray(self._positions.detach().cpu().numpy())
        vcol = None if self._colors is None else np.ascontiguousarray(self._colors.detach().cpu().numpy())
        ccol = None if self._cell_colors is None else np.ascontiguousarray(self._cell_colors.detach().cpu().numpy())
        res = ctypes.c_void_p()
        _lib.call("dtv_mesh_subdivide_vertices", cells.ctypes.data, cells.shape[0], pos.ctypes.data, V,
                  None if vcol is None else vcol.ctypes.data, None if ccol is None else ccol.ctypes.data,
                  order.ctypes.data, order.shape[0], ctypes.c_float(0.5), ctypes.byref(res))
        try:
            nt, nv = ctypes.c_uint64(), ctypes.c_uint64()
            _lib.call("dtv_split_result_sizes", res, ctypes.byref(nt), ctypes.byref(nv))
            c2 = np.empty((nt.value, 4), np.uint32)
            p2 = np.empty((nv.value, 3), np.float32)
            v2 = None if vcol is None else np.empty((nv.value, 4), np.float32)
            cc2 = None if ccol is None else np.empty((nt.value, 4), np.float32)
            _lib.call("dtv_split_result_copy", res, c2.ctypes.data, p2.ctypes.data,
                      None if v2 is None else v2.ctypes.data, None if cc2 is None else cc2.ctypes.data)
        finally:
            _lib.load().dtv_split_result_destroy(res)
        if cc2 is not None:
            self.set_tet_mesh_data_cell(c2, p2, cc2)
        else:
            self.set_tet_mesh_data(c2, p2, v2)
        if volume_renderer is not None:
            volume_renderer.set_tet_mesh(self)

    def set_force_use_ovm_representation(self) -> None:
        """TetMesh::setForceUseOvmRepresentation (Module.cpp:794): the
        reference keeps an OpenVolumeMesh copy of the mesh for coarse-to-fine
        splitting.  The split here works on the plain cell and vertex arrays
        (dtv_mesh_subdivide_vertices), so the flag is only recorded."""
        self._force_ovm = True

    # -- topology edits (Module.cpp:816-819) ---------------------------------
    def _host_arrays(self):
        pos = self._positions.detach().cpu().numpy()
        vcol = None if self._colors is None else self._colors.detach().cpu().numpy()
        ccol = None if self._cell_colors is None else self._cell_colors.detach().cpu().numpy()
        return pos, vcol, ccol

    def unlink_tets(self) -> None:
        """TetMesh::unlinkTets (TetMesh.cpp:1950-1989): every cell gets its
        own four vertices (a shared-index mesh becomes a cell soup)."""
        if self._cells is None:
            raise RuntimeError("Missing valid tet mesh.")
        pos, vcol, ccol = self._host_arrays()
        cells, pos, vcol = unlink_cells(self._cells, pos, vcol)
        if ccol is not None:
            self.set_tet_mesh_data_cell(cells, pos, ccol)
        else:
            self.set_tet_mesh_data(cells, pos, vcol)

    def remove_transparent_tets(self, alpha_threshold: float) -> None:
        """TetMesh::removeTransparentTets (TetMesh.cpp:1991-2084): removes the
        cells with no vertex alpha (per-cell colours: no cell alpha) >=
        alpha_threshold, and the vertices no remaining cell uses."""
        if self._cells is None:
            raise RuntimeError("Missing valid tet mesh.")
        pos, vcol, ccol = self._host_arrays()
        cells, pos, vcol, ccol = remove_transparent_cells(self._cells, pos, vcol, ccol, alpha_threshold)
        if ccol is not None:
            self.set_tet_mesh_data_cell(cells, pos, ccol)
        else:
            self.set_tet_mesh_data(cells, pos, vcol)

    # -- files (Module.cpp:787-788) ------------------------------------------
    def load_from_file(self, file_path: str) -> bool:
        """TetMesh::loadFromFile (TetMesh.cpp:1084-1150): .bintet files; False
        (with a warning) for an unsupported extension or an unreadable file."""
        import warnings

        from .mesh_io import SUPPORTED_EXTENSIONS, file_extension, read_bintet
        ext = file_extension(file_path)
        if ext not in SUPPORTED_EXTENSIONS:
            warnings.warn(f"Error in TetMesh.load_from_file: Unsupported file extension '.{ext}'.")
            return False
        try:
            cells, pos, vcol, ccol, _ = read_bintet(file_path)
        except RuntimeError as e:
            warnings.warn(f"Error in TetMesh.load_from_file: {e}")
            return False
        if vcol.shape[0] > 0:
            self.set_tet_mesh_data(cells, pos, vcol)
        if ccol is not None and ccol.shape[0] > 0:
            self.set_tet_mesh_data_cell(cells, pos, ccol)
        return True

    def save_to_file(self, file_path: str) -> bool:
        """TetMesh::saveToFile (TetMesh.cpp:1152-1173): .bintet (version 1 with
        vertex colours, version 2 with cell colours)."""
        from .mesh_io import SUPPORTED_EXTENSIONS, file_extension, write_bintet
        ext = file_extension(file_path)
        if ext not in SUPPORTED_EXTENSIONS:
            raise RuntimeError(
                f"Error in TetMeshData::createTetMeshWriterByExtension: Unsupported file extension '.{ext}'.")
        pos = self._positions.detach().cpu().numpy()
        vcol = None if self._colors is None else self._colors.detach().cpu().numpy()
        ccol = None if self._cell_colors is None else self._cell_colors.detach().cpu().numpy()
        write_bintet(file_path, self._cells, pos, vcol, ccol)
        return True

    # -- accessors ---------------------------------------------------------
    def get_num_cells(self) -> int:
        return 0 if self._cells is None else int(self._cells.shape[0])

    def get_num_vertices(self) -> int:
        return 0 if self._positions is None else int(self._positions.shape[0])

    def get_num_faces(self) -> int:
        return 0 if self._native is None else int(self._native.num_faces)

    def get_vertex_positions(self) -> torch.Tensor:
        return self._positions

    def get_vertex_colors(self) -> torch.Tensor:
        return self._colors

    def get_cell_colors(self) -> torch.Tensor:
        """Per-cell RGBA [T, 4] (ColorStorage.PER_CELL meshes; None otherwise)."""
        return self._cell_colors

    def get_cells(self) -> np.ndarray:
        return self._cells

    def get_vertex_boundary_bit_tensor(self) -> torch.Tensor:
        return self._vertex_boundary

    def get_color_storage(self) -> ColorStorage:
        return self._color_storage

    def get_bounding_box(self) -> AABB3:
        p = self._positions.detach()
        mn = p.min(dim=0).values.tolist()
        mx = p.max(dim=0).values.tolist()
        return AABB3(vec3(*mn), vec3(*mx))

    def get_is_empty(self) -> bool:
        return self._cells is None or self._cells.shape[0] == 0

    def set_vertices_changed(self, vertices_changed: bool = True) -> None:
        """No-op: renders read the position / colour tensors directly."""

    def on_zero_grad(self) -> None:
        """No-op on CUDA (the reference uses it for its CPU device path)."""

    def check_is_any_tet_degenerate(self) -> bool:
        """TetMesh::checkIsAnyTetDegenerate (TetMesh.cpp:544-558): valid tets have
        dot(cross(p1-p0, p2-p0), p3-p0) < 0."""
        p = self._positions.detach().double()
        c = torch.as_tensor(self._cells.astype(np.int64), device=p.device)
        p0, p1, p2, p3 = (p[c[:, k]] for k in range(4))
        vol = torch.sum(torch.cross(p1 - p0, p2 - p0, dim=1) * (p3 - p0), dim=1)
        return bool((vol >= 0).any().item())

    @property
    def native(self) -> NativeMesh:
        if self._native is None:
            raise RuntimeError("Missing valid tet mesh.")
        return self._native


def cube_central_gradient_data():
    """CUBE_CENTRAL_GRADIENT fixture (createBaseCubeHex, TetMesh.cpp:969-1014, scaled
    by 1/16 in loadTestData :1066-1076): 4 hexes, red denser central slab."""
    width = 4.0
    ml, mr = -width * 0.5, width * 0.5
    pos = np.array([
        [-4, -4, 4], [ml, -4, 4], [0, -4, 4], [mr, -4, 4], [4, -4, 4],
        [4, -4, -4], [mr, -4, -4], [0, -4, -4], [ml, -4, -4], [-4, -4, -4],
        [-4, 4, 4], [ml, 4, 4], [0, 4, 4], [mr, 4, 4], [4, 4, 4],
        [4, 4, -4], [mr, 4, -4], [0, 4, -4], [ml, 4, -4], [-4, 4, -4],
    ], dtype=np.float32) * np.float32(1.0 / 16.0)
    alpha_scale = 0.25
    c0 = [0.5, 0.5, 0.5, 0.0625 * alpha_scale]
    c1 = [1.0, 0.0, 0.0, 0.125 * alpha_scale]
    col = np.array([c0, c0, c1, c0, c0] * 4, dtype=np.float32)
    hexes = np.array([
        9, 8, 18, 19, 0, 1, 11, 10,
        8, 7, 17, 18, 1, 2, 12, 11,
        7, 6, 16, 17, 2, 3, 13, 12,
        6, 5, 15, 16, 3, 4, 14, 13,
    ], dtype=np.uint32)
    return convert_hex_to_tet_indices(hexes), pos, col
