"""ctypes binding of the C ABI in include/difftetvr_b200.h.

The shared library is built in-tree (difftetvr_b200/libdifftetvr_b200.so, see
build.py).  There is no CPU fallback: if the library is missing or cannot be
loaded, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "libdifftetvr_b200.so")

DTV_OK = 0
DTV_ERR_ARG = 1
DTV_ERR_BUDGET = 2
DTV_ERR_CUDA = 3
DTV_ERR_TIMEOUT = 4
DTV_ERR_STATE = 5
DTV_OVER_BUDGET_ERROR = 0
DTV_OVER_BUDGET_RECOMPUTE = 1

_ERR_NAMES = {
    DTV_ERR_ARG: "DTV_ERR_ARG",
    DTV_ERR_BUDGET: "DTV_ERR_BUDGET",
    DTV_ERR_CUDA: "DTV_ERR_CUDA",
    DTV_ERR_TIMEOUT: "DTV_ERR_TIMEOUT",
    DTV_ERR_STATE: "DTV_ERR_STATE",
}

c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_vp = ctypes.c_void_p


class Camera(ctypes.Structure):
    _fields_ = [
        ("view", ctypes.c_float * 16),
        ("fovy", ctypes.c_float),
        ("znear", ctypes.c_float),
        ("zfar", ctypes.c_float),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("composite_tile", ctypes.c_int32),
        ("adjoint_tile", ctypes.c_int32),
        ("sort_surrogate_classes", ctypes.c_uint32),
        ("sort_bucket_classes", ctypes.c_uint32),
    ]


class RenderParams(ctypes.Structure):
    _fields_ = [
        ("attenuation", ctypes.c_float),
        ("use_early_ray_termination", ctypes.c_int32),
        ("early_ray_out_thresh", ctypes.c_float),
        ("clear_color", ctypes.c_float * 4),
        ("use_abs_grad", ctypes.c_int32),
        ("over_budget", ctypes.c_int32),
        ("fragment_budget_bytes", ctypes.c_uint64),
    ]


class BatchView(ctypes.Structure):
    _fields_ = [
        ("mesh", ctypes.c_int32),
        ("grad_slot", ctypes.c_int32),
        ("camera", Camera),
        ("d_image", ctypes.c_void_p),
        ("d_target", ctypes.c_void_p),
        ("d_image_adjoint", ctypes.c_void_p),
    ]


class BatchGradSlot(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_int32), ("d_grad_positions", ctypes.c_void_p), ("d_grad_colors", ctypes.c_void_p)]


class BatchOptim(ctypes.Structure):
    _fields_ = [
        ("lr_positions", ctypes.c_float),
        ("lr_colors", ctypes.c_float),
        ("beta1", ctypes.c_float),
        ("beta2", ctypes.c_float),
        ("eps", ctypes.c_float),
        ("clamp_colors", ctypes.c_int32),
        ("fixed_boundary", ctypes.c_int32),
    ]


class DtvError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {message}")
        self.code = code


# Exported symbols: name -> (restype, argtypes).
SIGNATURES = {
    "dtv_version": (ctypes.c_int32, []),
    "dtv_last_error_string": (ctypes.c_char_p, []),
    "dtv_build_hex_mesh": (ctypes.c_int32, [c_f32p, c_f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            c_vp, c_vp]),
    "dtv_mesh_build_faces_host": (ctypes.c_int32, [c_vp, ctypes.c_uint64, ctypes.c_uint64, c_vp, c_vp, c_vp, c_vp,
                                                   c_u64p]),
    "dtv_mesh_create": (ctypes.c_int32, [c_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(c_vp)]),
    "dtv_mesh_destroy": (ctypes.c_int32, [c_vp]),
    "dtv_mesh_get_info": (ctypes.c_int32, [c_vp, c_u64p, c_u64p, c_u64p]),
    "dtv_mesh_copy_faces": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dtv_mesh_vertex_boundary_device": (ctypes.c_int32, [c_vp, ctypes.POINTER(c_vp)]),
    "dtv_renderer_create": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(c_vp)]),
    "dtv_renderer_destroy": (ctypes.c_int32, [c_vp]),
    "dtv_renderer_render": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(Camera),
                                             ctypes.POINTER(RenderParams), c_vp, c_vp]),
    "dtv_renderer_render_adjoint": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, c_vp, c_vp,
                                                     c_vp]),
    "dtv_batch_reserve": (ctypes.c_int32, [c_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_uint64, c_vp]),
    "dtv_renderer_render_cells": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(Camera),
                                                   ctypes.POINTER(RenderParams), c_vp, c_vp]),
    "dtv_renderer_render_adjoint_cells": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, c_vp,
                                                           c_vp, c_vp]),
    "dtv_renderer_get_num_fragments": (ctypes.c_int32, [c_vp, c_u64p]),
    "dtv_renderer_set_tuning": (ctypes.c_int32, [c_vp, ctypes.POINTER(Tuning)]),
    "dtv_renderer_get_tuning": (ctypes.c_int32, [c_vp, ctypes.POINTER(Tuning)]),
    "dtv_batch_set_tuning": (ctypes.c_int32, [c_vp, ctypes.POINTER(Tuning)]),
    "dtv_batch_get_tuning": (ctypes.c_int32, [c_vp, ctypes.POINTER(Tuning)]),
    "dtv_renderer_get_num_bands": (ctypes.c_int32, [c_vp, ctypes.POINTER(ctypes.c_int32)]),
    "dtv_mesh_subdivide_vertices": (ctypes.c_int32, [c_vp, ctypes.c_uint64, c_vp, ctypes.c_uint64, c_vp, c_vp, c_vp,
                                                     ctypes.c_uint64, ctypes.c_float, ctypes.POINTER(c_vp)]),
    "dtv_split_result_sizes": (ctypes.c_int32, [c_vp, c_u64p, c_u64p]),
    "dtv_split_result_copy": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dtv_split_result_destroy": (ctypes.c_int32, [c_vp]),
    "dtv_bintet_peek": (ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint32), c_u64p, c_u64p, c_u64p,
                                          c_u64p]),
    "dtv_bintet_read": (ctypes.c_int32, [ctypes.c_char_p, c_vp, c_vp, c_vp, c_vp]),
    "dtv_bintet_write": (ctypes.c_int32, [ctypes.c_char_p, c_vp, ctypes.c_uint64, c_vp, ctypes.c_uint64, c_vp,
                                           ctypes.c_uint64, c_vp, ctypes.c_uint64]),
    "dtv_tet_regularizer_grad": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_float, ctypes.c_float, c_vp, c_vp, c_vp]),
    "dtv_renderer_copy_fragments": (ctypes.c_int32, [c_vp, c_vp, c_vp, ctypes.c_uint64, c_vp]),
    "dtv_renderer_copy_pixel_state": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp]),
    "dtv_renderer_set_timing": (ctypes.c_int32, [c_vp, ctypes.c_int32]),
    "dtv_renderer_stage_times": (ctypes.c_int32, [c_vp, c_f32p, ctypes.c_int32]),
    "dtv_render_noalloc": (ctypes.c_int32, [c_vp, c_vp, c_vp, ctypes.POINTER(Camera), ctypes.POINTER(RenderParams),
                                            c_vp, c_vp]),
    "dtv_batch_create": (ctypes.c_int32, [ctypes.POINTER(c_vp)]),
    "dtv_batch_destroy": (ctypes.c_int32, [c_vp]),
    "dtv_batch_set_meshes": (ctypes.c_int32, [c_vp, ctypes.c_int32, c_vp, c_vp, c_vp]),
    "dtv_batch_render": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.POINTER(BatchView), ctypes.POINTER(RenderParams),
                                          c_vp]),
    "dtv_batch_render_async": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.POINTER(BatchView),
                                                ctypes.POINTER(RenderParams), c_vp]),
    "dtv_batch_render_status": (ctypes.c_int32, [c_vp, ctypes.POINTER(ctypes.c_int32), c_u64p]),
    "dtv_batch_render_adjoint": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.POINTER(BatchView), ctypes.c_int32,
                                                  ctypes.POINTER(BatchGradSlot), ctypes.c_int32, c_vp]),
    "dtv_batch_train_step": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.POINTER(BatchView),
                                              ctypes.POINTER(RenderParams), ctypes.POINTER(BatchOptim), c_vp, c_vp]),
    "dtv_batch_set_graph": (ctypes.c_int32, [c_vp, ctypes.c_int32]),
    "dtv_batch_get_info": (ctypes.c_int32, [c_vp, c_u64p, c_u64p, c_u64p, ctypes.POINTER(ctypes.c_int32)]),
    "dtv_loss_l2": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_uint64, ctypes.c_float, c_vp, c_vp, c_vp]),
    "dtv_adam_step": (ctypes.c_int32, [c_vp, c_vp, c_vp, c_vp, ctypes.c_uint64, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_int32, c_vp,
                                       ctypes.c_int32, ctypes.c_int32, c_vp]),
}

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load the CUDA library (once).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"difftetvr_b200 CUDA library not found at {LIB_PATH}; build it with "
                "`python -m difftetvr_b200.build` (there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(code: int) -> None:
    if code != DTV_OK:
        msg = load().dtv_last_error_string()
        raise DtvError(code, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
