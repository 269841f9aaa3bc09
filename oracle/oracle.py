"""ctypes wrapper of the CPU oracle (oracle/dtv_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker / timed CPU port.  The product
package difftetvr_b200 never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_DIR, "liboracle.so")
_lib = None

_vp = ctypes.c_void_p


class Camera(ctypes.Structure):
    _fields_ = [("view", ctypes.c_float * 16), ("fovy", ctypes.c_float), ("znear", ctypes.c_float),
                ("zfar", ctypes.c_float), ("width", ctypes.c_int32), ("height", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [("attenuation", ctypes.c_float), ("use_ert", ctypes.c_int32), ("ert_thresh", ctypes.c_float),
                ("clear_color", ctypes.c_float * 4), ("use_abs_grad", ctypes.c_int32),
                ("row_begin", ctypes.c_int32), ("row_end", ctypes.c_int32)]


def build() -> str:
    """Compile liboracle.so with the Makefile next to this file (if out of date)."""
    src = os.path.join(_DIR, "dtv_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        env = dict(os.environ)
        env.pop("CXX", None)
        env.pop("CC", None)
        subprocess.run(["make", "-C", _DIR, "liboracle.so"], check=True, env=env, capture_output=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.orc_build_faces.restype = ctypes.c_int64
        lib.orc_build_faces.argtypes = [_vp, ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp, _vp]
        lib.orc_fragments.restype = ctypes.c_int64
        lib.orc_fragments.argtypes = [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.POINTER(Camera), _vp,
                                      _vp, ctypes.c_int64]
        lib.orc_fragments_rows.restype = ctypes.c_int64
        lib.orc_fragments_rows.argtypes = [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.POINTER(Camera),
                                           ctypes.c_int32, ctypes.c_int32, _vp, _vp, ctypes.c_int64]
        lib.orc_project_f32.restype = None
        lib.orc_project_f32.argtypes = [_vp, ctypes.c_int64, ctypes.POINTER(Camera), _vp, _vp, _vp]
        for name in ("orc_render_f64", "orc_render_f32"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, ctypes.POINTER(Camera),
                           ctypes.POINTER(Params), _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int64)]
        for name in ("orc_adjoint_f64", "orc_adjoint_f32"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, ctypes.POINTER(Camera),
                           ctypes.POINTER(Params), _vp, _vp, _vp]
        lib.orc_render_frozen_f64.restype = ctypes.c_int
        lib.orc_render_frozen_f64.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int64,
                                              ctypes.POINTER(Camera), ctypes.POINTER(Params), _vp]
        lib.orc_refmode_f64.restype = ctypes.c_int
        lib.orc_refmode_f64.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int64,
                                        ctypes.POINTER(Camera), ctypes.POINTER(Params), _vp, _vp, _vp, _vp, _vp,
                                        ctypes.c_int32]
        lib.orc_refmode_bary_uv.restype = None
        lib.orc_refmode_bary_uv.argtypes = [_vp] * 8
        lib.orc_tet_faces.restype = None
        lib.orc_tet_faces.argtypes = [_vp, ctypes.c_int64, _vp]
        for name in ("orc_raytet_f64", "orc_raytet_f32"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, ctypes.POINTER(Camera),
                           ctypes.POINTER(Params), _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        lib.orc_segment_integral.restype = None
        lib.orc_segment_integral.argtypes = [ctypes.c_double, _vp, _vp, ctypes.c_double, _vp]
        lib.orc_num_threads.restype = ctypes.c_int
        lib.orc_cells_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, ctypes.c_int64,
                                      ctypes.POINTER(Camera), ctypes.POINTER(Params), _vp, _vp, _vp, _vp, _vp, _vp,
                                      _vp, _vp]
        lib.orc_cells_f64.restype = ctypes.c_int
        lib.orc_tet_regularizer.argtypes = [_vp, ctypes.c_int64, _vp, ctypes.c_double, ctypes.c_double, _vp]
        lib.orc_tet_regularizer.restype = ctypes.c_double
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def make_camera(view, fovy, width, height, znear=0.01, zfar=100.0) -> Camera:
    c = Camera()
    c.view[:] = [float(v) for v in view]
    c.fovy, c.znear, c.zfar = float(fovy), float(znear), float(zfar)
    c.width, c.height = int(width), int(height)
    return c


def make_params(attenuation=1.0, use_ert=False, ert_thresh=1e-4, clear=(0, 0, 0, 0), use_abs_grad=False,
                rows=None) -> Params:
    p = Params()
    p.attenuation = float(attenuation)
    p.use_ert = int(bool(use_ert))
    p.ert_thresh = float(ert_thresh)
    p.clear_color[:] = [float(c) for c in clear]
    p.use_abs_grad = int(bool(use_abs_grad))
    p.row_begin, p.row_end = (0, 0) if rows is None else (int(rows[0]), int(rows[1]))
    return p


class Faces:
    """buildFacesSlim restatement output."""

    def __init__(self, cells: np.ndarray, num_vertices: int):
        lib = load()
        cells = np.ascontiguousarray(cells, dtype=np.uint32).reshape(-1, 4)
        T = cells.shape[0]
        tri = np.empty(12 * T, np.uint32)
        fb = np.empty(4 * T, np.uint32)
        f2t = np.empty(8 * T, np.uint32)
        vb = np.empty(num_vertices, np.uint32)
        F = lib.orc_build_faces(_p(cells), T, num_vertices, _p(tri), _p(fb), _p(f2t), _p(vb))
        self.tri = tri[:3 * F].reshape(F, 3).copy()
        self.face_boundary = fb[:F].copy()
        self.face_to_tet = f2t[:2 * F].reshape(F, 2).copy()
        self.vertex_boundary = vb
        self.num_faces = F
        self.tet_faces = np.empty(4 * T, np.uint32)
        lib.orc_tet_faces(_p(cells), T, _p(self.tet_faces))


def fragments(faces: Faces, positions: np.ndarray, cam: Camera):
    """(offsets i64[P+1], records u64[Nf]) sorted per pixel."""
    lib = load()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    P = cam.width * cam.height
    off = np.empty(P + 1, np.int64)
    nf = lib.orc_fragments(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pos), pos.shape[0],
                           ctypes.byref(cam), _p(off), None, 0)
    rec = np.empty(max(nf, 1), np.uint64)
    lib.orc_fragments(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pos), pos.shape[0],
                      ctypes.byref(cam), _p(off), _p(rec), rec.shape[0])
    return off, rec[:nf]


def fragments_rows(faces: Faces, positions: np.ndarray, cam: Camera, row_begin: int, row_end: int):
    """fragments() restricted to pixel rows [row_begin, row_end): offsets i64[P+1]
    (empty lists outside the rows), records u64 of those rows."""
    lib = load()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    P = cam.width * cam.height
    off = np.empty(P + 1, np.int64)
    args = (_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pos), pos.shape[0], ctypes.byref(cam),
            int(row_begin), int(row_end), _p(off))
    nf = lib.orc_fragments_rows(*args, None, 0)
    rec = np.empty(max(nf, 1), np.uint64)
    lib.orc_fragments_rows(*args, _p(rec), rec.shape[0])
    return off, rec[:nf]


def project_f32(positions: np.ndarray, cam: Camera):
    lib = load()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    V = pos.shape[0]
    sxy = np.empty((V, 3), np.float32)
    xy = np.empty((V, 2), np.int32)
    valid = np.empty(V, np.uint8)
    lib.orc_project_f32(_p(pos), V, ctypes.byref(cam), _p(sxy), _p(xy), _p(valid))
    return sxy, xy, valid.astype(bool)


def render(faces: Faces, positions, colors, cam: Camera, prm: Params, precision: int = 64):
    """Forward composite.  Returns (image [H,W,4], T_final [H,W], termination [H,W], Nf)."""
    lib = load()
    dt = np.float64 if precision == 64 else np.float32
    pos = np.ascontiguousarray(positions, dtype=dt)
    col = np.ascontiguousarray(colors, dtype=dt)
    P = cam.width * cam.height
    img = np.zeros((P, 4), dt)
    tf = np.ones(P, dt)
    term = np.zeros(P, np.uint32)
    nf = ctypes.c_int64(0)
    fn = lib.orc_render_f64 if precision == 64 else lib.orc_render_f32
    fn(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pos), _p(col), pos.shape[0],
       ctypes.byref(cam), ctypes.byref(prm), _p(img), _p(tf), _p(term), ctypes.byref(nf))
    H, W = cam.height, cam.width
    return img.reshape(H, W, 4), tf.reshape(H, W), term.reshape(H, W), int(nf.value)


def render_frozen(faces: Faces, positions_coverage, positions, colors, cam: Camera, prm: Params):
    """FP64 forward whose fragment lists come from positions_coverage (float32)."""
    lib = load()
    pc = np.ascontiguousarray(positions_coverage, dtype=np.float32)
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    col = np.ascontiguousarray(colors, dtype=np.float64)
    img = np.zeros((cam.width * cam.height, 4), np.float64)
    lib.orc_render_frozen_f64(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pc), _p(pos), _p(col),
                              pos.shape[0], ctypes.byref(cam), ctypes.byref(prm), _p(img))
    return img.reshape(cam.height, cam.width, 4)


def adjoint(faces: Faces, positions, colors, cam: Camera, prm: Params, image_adjoint, precision: int = 64):
    """Exact adjoint.  Returns (grad_positions [V,3], grad_colors [V,4])."""
    lib = load()
    dt = np.float64 if precision == 64 else np.float32
    pos = np.ascontiguousarray(positions, dtype=dt)
    col = np.ascontiguousarray(colors, dtype=dt)
    gimg = np.ascontiguousarray(image_adjoint, dtype=dt).reshape(-1, 4)
    gp = np.zeros((pos.shape[0], 3), dt)
    gc = np.zeros((pos.shape[0], 4), dt)
    fn = lib.orc_adjoint_f64 if precision == 64 else lib.orc_adjoint_f32
    fn(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pos), _p(col), pos.shape[0],
       ctypes.byref(cam), ctypes.byref(prm), _p(gimg), _p(gp), _p(gc))
    return gp, gc


def raytet(faces: Faces, positions, colors, cam: Camera, prm: Params, image_adjoint=None, precision: int = 64,
           positions_coverage=None):
    """Ray-tet (intersection) path: returns (image [H,W,4], T_final [H,W], segments [H,W]) and, with
    image_adjoint, also (grad_positions [V,3], grad_colors [V,4])."""
    lib = load()
    dt = np.float64 if precision == 64 else np.float32
    pos = np.ascontiguousarray(positions, dtype=dt)
    col = np.ascontiguousarray(colors, dtype=dt)
    P = cam.width * cam.height
    img = np.zeros((P, 4), dt)
    tf = np.ones(P, dt)
    nseg = np.zeros(P, np.uint32)
    V = pos.shape[0]
    gp = np.zeros((V, 3), dt)
    gc = np.zeros((V, 4), dt)
    gimg = None if image_adjoint is None else np.ascontiguousarray(image_adjoint, dtype=dt).reshape(-1, 4)
    pc = None if positions_coverage is None else np.ascontiguousarray(positions_coverage, dtype=np.float32)
    fn = lib.orc_raytet_f64 if precision == 64 else lib.orc_raytet_f32
    fn(_p(faces.tri), _p(faces.face_boundary), _p(faces.face_to_tet), _p(faces.tet_faces), faces.num_faces,
       _p(pos), _p(col), V, ctypes.byref(cam), ctypes.byref(prm), _p(img), _p(tf), _p(nseg),
       None if gimg is None else _p(gimg), _p(gp), _p(gc), None if pc is None else _p(pc))
    H, W = cam.height, cam.width
    out = (img.reshape(H, W, 4), tf.reshape(H, W), nseg.reshape(H, W))
    return out if gimg is None else out + (gp, gc)


def refmode(faces: Faces, positions, colors, cam: Camera, prm: Params, image_adjoint=None, skip0: bool = True):
    """The reference's own formulas (dtv_oracle.cpp, namespace refmode) on this
    oracle's fragment sets: (image [H,W,4], termination [H,W]) and, with
    image_adjoint, also the reference adjoint's (grad_positions [V,3],
    grad_colors [V,4]).  FP64 except the FP32 depth-buffer value.  skip0=False
    differentiates all four sub-segments (the reference skips the first)."""
    lib = load()
    pf = np.ascontiguousarray(positions, dtype=np.float32)
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    col = np.ascontiguousarray(colors, dtype=np.float64)
    V = pos.shape[0]
    P = cam.width * cam.height
    img = np.zeros((P, 4))
    term = np.zeros(P, np.uint32)
    gimg = None if image_adjoint is None else np.ascontiguousarray(image_adjoint, np.float64).reshape(-1, 4)
    gp = np.zeros((V, 3))
    gc = np.zeros((V, 4))
    lib.orc_refmode_f64(_p(faces.tri), _p(faces.face_boundary), faces.num_faces, _p(pf), _p(pos), _p(col), V,
                        ctypes.byref(cam), ctypes.byref(prm), _p(img), _p(term),
                        None if gimg is None else _p(gimg), _p(gp), _p(gc), int(bool(skip0)))
    H, W = cam.height, cam.width
    out = (img.reshape(H, W, 4), term.reshape(H, W))
    return out if gimg is None else out + (gp, gc)


def refmode_bary_uv(p, p0, p1, p2):
    """(u, v, du [3,3], dv [3,3]) of the reference mode's unsigned weights of
    world point p on face (p0, p1, p2), gradients w.r.t. the vertices."""
    lib = load()
    arr = [np.ascontiguousarray(x, np.float64) for x in (p, p0, p1, p2)]
    u, v = np.zeros(1), np.zeros(1)
    du, dv = np.zeros(9), np.zeros(9)
    lib.orc_refmode_bary_uv(*[_p(a) for a in arr], _p(u), _p(v), _p(du), _p(dv))
    return float(u[0]), float(v[0]), du.reshape(3, 3), dv.reshape(3, 3)


def segment_integral(t, c0, c1, a):
    lib = load()
    c0 = np.ascontiguousarray(c0, np.float64)
    c1 = np.ascontiguousarray(c1, np.float64)
    out = np.zeros(4, np.float64)
    lib.orc_segment_integral(float(t), _p(c0), _p(c1), float(a), _p(out))
    return out


def render_cells(faces: Faces, positions, cell_colors, cam: Camera, prm: Params, image_adjoint=None,
                 positions_coverage=None):
    """Per-cell colours (ColorStorage.PER_CELL), FP64: (image [H,W,4], T_final, termination, #fragments) and,
    with image_adjoint, also (grad_positions [V,3], grad_cell_colors [T,4])."""
    lib = load()
    pos = np.ascontiguousarray(positions, np.float64)
    ccol = np.ascontiguousarray(cell_colors, np.float64)
    V, T = pos.shape[0], ccol.shape[0]
    P = cam.width * cam.height
    img = np.zeros((P, 4))
    tf = np.ones(P)
    term = np.zeros(P, np.uint32)
    nf = ctypes.c_int64()
    gp = np.zeros((V, 3))
    gc = np.zeros((T, 4))
    gimg = None if image_adjoint is None else np.ascontiguousarray(image_adjoint, np.float64).reshape(-1, 4)
    pc = None if positions_coverage is None else np.ascontiguousarray(positions_coverage, np.float32)
    lib.orc_cells_f64(_p(faces.tri), _p(faces.face_boundary), _p(faces.face_to_tet), faces.num_faces, _p(pos),
                      _p(ccol), V, T, ctypes.byref(cam), ctypes.byref(prm), _p(img), _p(tf), _p(term),
                      ctypes.byref(nf), None if gimg is None else _p(gimg), _p(gp), _p(gc),
                      None if pc is None else _p(pc))
    H, W = cam.height, cam.width
    out = (img.reshape(H, W, 4), tf.reshape(H, W), term.reshape(H, W), int(nf.value))
    return out if gimg is None else out + (gp, gc)


def tet_regularizer(cells, positions, reg_lambda: float, softplus_beta: float):
    """FP64 tet-quality regularizer: (penalty summed over tets, gradient [V,3])."""
    lib = load()
    cells = np.ascontiguousarray(cells, np.uint32)
    pos = np.ascontiguousarray(positions, np.float64)
    grad = np.zeros_like(pos)
    total = lib.orc_tet_regularizer(_p(cells), cells.shape[0], _p(pos), float(reg_lambda), float(softplus_beta),
                                    _p(grad))
    return float(total), grad


def num_threads() -> int:
    return int(load().orc_num_threads())
