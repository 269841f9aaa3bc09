"""Coarse-to-fine subdivision (dtv_mesh_subdivide_vertices) on the CPU: the
refined mesh is conforming (every face shared by at most two tets, the
boundary surface unchanged), keeps the volume and the orientation of every
tet, interpolates vertex colours on the split edges and inherits cell
colours."""
import ctypes

import numpy as np
import pytest

from difftetvr_b200 import _lib
from difftetvr_b200 import synthetic as S
from difftetvr_b200.tet_mesh import build_faces_host


def subdivide(cells, pos, split, vcol=None, ccol=None, t=0.5):
    cells = np.ascontiguousarray(cells, np.uint32)
    pos = np.ascontiguousarray(pos, np.float32)
    split = np.ascontiguousarray(split, np.uint32)
    res = ctypes.c_void_p()
    _lib.call("dtv_mesh_subdivide_vertices", cells.ctypes.data, cells.shape[0], pos.ctypes.data, pos.shape[0],
              None if vcol is None else np.ascontiguousarray(vcol, np.float32).ctypes.data,
              None if ccol is None else np.ascontiguousarray(ccol, np.float32).ctypes.data,
              split.ctypes.data, split.shape[0], ctypes.c_float(t), ctypes.byref(res))
    nt, nv = ctypes.c_uint64(), ctypes.c_uint64()
    _lib.call("dtv_split_result_sizes", res, ctypes.byref(nt), ctypes.byref(nv))
    c2 = np.empty((nt.value, 4), np.uint32)
    p2 = np.empty((nv.value, 3), np.float32)
    v2 = np.empty((nv.value, 4), np.float32)
    cc2 = np.empty((nt.value, 4), np.float32)
    _lib.call("dtv_split_result_copy", res, c2.ctypes.data, p2.ctypes.data, v2.ctypes.data, cc2.ctypes.data)
    _lib.load().dtv_split_result_destroy(res)
    return c2, p2, (v2 if vcol is not None else None), (cc2 if ccol is not None else None)


def dets(cells, pos):
    p = pos.astype(np.float64)[cells.astype(np.int64)]
    return np.linalg.det(np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=1))


def boundary_area(cells, pos):
    tri, fb, f2t, vb = build_faces_host(cells, pos.shape[0])
    t = tri[fb.astype(bool)].astype(np.int64)
    p = pos.astype(np.float64)
    return 0.5 * np.linalg.norm(np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]]), axis=1).sum()


def assert_conforming(cells, pos):
    faces = np.sort(cells[:, [[0, 1, 2], [1, 0, 3], [0, 2, 3], [2, 1, 3]]].reshape(-1, 3), axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    assert counts.max() <= 2


@pytest.mark.parametrize("n,frac,seed", [(3, 0.02, 1), (4, 0.15, 2), (5, 0.4, 3)])
def test_refinement_is_conforming_and_keeps_volume(n, frac, seed):
    cells, pos = S.kuhn_mesh(n, seed=seed)
    rng = np.random.default_rng(seed)
    split = rng.choice(pos.shape[0], size=max(1, int(frac * pos.shape[0])), replace=False)
    c2, p2, _, _ = subdivide(cells, pos, split)
    d0, d1 = dets(cells, pos), dets(c2, p2)
    assert np.all(d0 < 0) and np.all(d1 < 0)  # the Kuhn cells' orientation, kept by every new tet
    np.testing.assert_allclose(np.abs(d1).sum(), np.abs(d0).sum(), rtol=1e-6)
    assert_conforming(c2, p2)
    np.testing.assert_allclose(boundary_area(c2, p2), boundary_area(cells, pos), rtol=1e-6)
    assert c2.shape[0] > cells.shape[0] and p2.shape[0] > pos.shape[0]
    # Old vertices keep their index and position.
    np.testing.assert_array_equal(p2[:pos.shape[0]], pos)


def test_single_vertex_counts_and_colours():
    cells, pos = S.kuhn_mesh(2, seed=0, jitter=0.0)
    v = 13  # the centre vertex of the 3x3x3 grid
    star = np.flatnonzero((cells == v).any(1))
    nbrs = np.unique(cells[star])
    nbrs = nbrs[nbrs != v]
    vcol = np.random.default_rng(0).uniform(size=(pos.shape[0], 4)).astype(np.float32)
    c2, p2, v2, _ = subdivide(cells, pos, [v], vcol=vcol)
    assert c2.shape[0] == cells.shape[0] + 3 * star.size
    assert p2.shape[0] == pos.shape[0] + nbrs.size
    # New vertices: edge midpoints in increasing order of the far vertex, colours interpolated.
    np.testing.assert_allclose(p2[pos.shape[0]:], 0.5 * (pos[v] + pos[nbrs]), rtol=0, atol=1e-7)
    np.testing.assert_allclose(v2[pos.shape[0]:], 0.5 * (vcol[v] + vcol[nbrs]), rtol=0, atol=1e-7)
    # Surviving tets first, in their old order.
    keep = np.setdiff1d(np.arange(cells.shape[0]), star)
    np.testing.assert_array_equal(c2[:keep.size], cells[keep])


def test_cell_colours_are_inherited_and_sequential_splits_compose():
    cells, pos = S.kuhn_mesh(3, seed=5)
    ccol = np.random.default_rng(1).uniform(size=(cells.shape[0], 4)).astype(np.float32)
    c2, p2, _, cc2 = subdivide(cells, pos, [21, 22, 26], ccol=ccol)
    # Every new tet lies inside one old tet and carries its colour: check by
    # the colour of the old tet containing the new tet's centroid.
    cen = p2[c2.astype(np.int64)].mean(1).astype(np.float64)
    p = pos.astype(np.float64)[cells.astype(np.int64)]
    T = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    Tinv = np.linalg.inv(T)
    for i in range(0, c2.shape[0], 7):
        lam = np.einsum("tij,tj->ti", Tinv, cen[i] - p[:, 0])
        inside = np.flatnonzero((lam > -1e-9).all(1) & (lam.sum(1) < 1 + 1e-9))
        assert inside.size == 1
        np.testing.assert_array_equal(cc2[i], ccol[inside[0]])
    assert_conforming(c2, p2)
    assert np.all(dets(c2, p2) < 0)


def test_errors():
    from difftetvr_b200._lib import DTV_ERR_ARG, DtvError
    cells, pos = S.kuhn_mesh(2, seed=0)
    with pytest.raises(DtvError) as e:
        subdivide(cells, pos, [pos.shape[0]])
    assert e.value.code == DTV_ERR_ARG
    with pytest.raises(DtvError):
        subdivide(cells, pos, [1], t=1.0)
