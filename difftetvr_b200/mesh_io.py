"""Tet mesh files.  `.bintet` (the reference's binary format,
src/Tet/Loaders/BinTetLoader.cpp:37-138) is read and written by the native
library (dtv_bintet_*); the arrays are plain numpy on the host."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

SUPPORTED_EXTENSIONS = ("bintet",)


def file_extension(path: str) -> str:
    return os.path.splitext(str(path))[1][1:].lower()


def peek_bintet(path: str) -> dict:
    """Header of a .bintet file: version and array sizes (BinTetLoader::peekSizes)."""
    ver = ctypes.c_uint32()
    t, v, vc, cc = (ctypes.c_uint64() for _ in range(4))
    _lib.call("dtv_bintet_peek", os.fsencode(path), ctypes.byref(ver), ctypes.byref(t), ctypes.byref(v),
              ctypes.byref(vc), ctypes.byref(cc))
    return {"version": int(ver.value), "num_cells": int(t.value), "num_vertices": int(v.value),
            "num_vertex_colors": int(vc.value), "num_cell_colors": int(cc.value)}


def read_bintet(path: str):
    """(cells u32[T,4], positions f32[V,3], vertex_colors f32[Nv,4], cell_colors f32[Nc,4] or None, version)."""
    h = peek_bintet(path)
    cells = np.empty((h["num_cells"], 4), np.uint32)
    pos = np.empty((h["num_vertices"], 3), np.float32)
    vcol = np.empty((h["num_vertex_colors"], 4), np.float32)
    ccol = np.empty((h["num_cell_colors"], 4), np.float32) if h["version"] == 2 else None
    _lib.call("dtv_bintet_read", os.fsencode(path), cells.ctypes.data, pos.ctypes.data, vcol.ctypes.data,
              None if ccol is None else ccol.ctypes.data)
    return cells, pos, vcol, ccol, h["version"]


def write_bintet(path: str, cells, positions, vertex_colors=None, cell_colors=None) -> None:
    """Version 1 (vertex colours) or, with cell colours, version 2 (BinTetWriter::saveToFile)."""
    cells = np.ascontiguousarray(np.asarray(cells, np.uint32).reshape(-1, 4))
    pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    vcol = np.zeros((0, 4), np.float32) if vertex_colors is None else \
        np.ascontiguousarray(np.asarray(vertex_colors, np.float32).reshape(-1, 4))
    ccol = np.zeros((0, 4), np.float32) if cell_colors is None else \
        np.ascontiguousarray(np.asarray(cell_colors, np.float32).reshape(-1, 4))
    _lib.call("dtv_bintet_write", os.fsencode(path), cells.ctypes.data, cells.shape[0], pos.ctypes.data,
              pos.shape[0], vcol.ctypes.data, vcol.shape[0], ccol.ctypes.data, ccol.shape[0])
