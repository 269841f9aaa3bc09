"""Host-side mesh preparation vs independent restatements (no GPU needed)."""
import numpy as np
import pytest

import difftetvr_b200 as d
from difftetvr_b200 import synthetic as S

HEX_TO_TET = np.array([[0, 4, 7, 6], [0, 4, 6, 5], [0, 3, 6, 7], [0, 3, 2, 6], [0, 1, 5, 6], [0, 1, 6, 2]])


def numpy_hex_mesh(xs, ys, zs, lo=-1.0, hi=1.0):
    """setHexMeshConst (TetMesh.cpp:1882-1936) restated with numpy."""
    iz, iy, ix = np.meshgrid(np.arange(zs), np.arange(ys), np.arange(xs), indexing="ij")
    f = lambda i, n: np.float32(lo) + (i.astype(np.float32) / np.float32(n - 1)) * np.float32(hi - lo)  # noqa: E731
    pos = np.stack([f(ix, xs), f(iy, ys), f(iz, zs)], -1).reshape(-1, 3).astype(np.float32)
    idx = lambda x, y, z: z * xs * ys + y * xs + x  # noqa: E731
    cells = []
    for z in range(zs - 1):
        for y in range(ys - 1):
            for x in range(xs - 1):
                hx = [idx(x, y, z), idx(x + 1, y, z), idx(x + 1, y + 1, z), idx(x, y + 1, z),
                      idx(x, y, z + 1), idx(x + 1, y, z + 1), idx(x + 1, y + 1, z + 1), idx(x, y + 1, z + 1)]
                for t in HEX_TO_TET:
                    cells.append([hx[k] for k in t])
    return np.array(cells, np.uint32), pos


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 4, 5), (9, 9, 9)])
def test_hex_mesh_matches_restatement(dims):
    cells, pos = d.build_hex_mesh((-1, -1, -1), (1, 1, 1), *dims)
    c2, p2 = numpy_hex_mesh(*dims)
    assert np.array_equal(cells, c2)
    assert np.array_equal(pos, p2)


@pytest.mark.parametrize("n", [1, 2, 8, 16])
def test_kuhn_face_counts_and_orientation(n):
    cells, pos = S.kuhn_mesh(n, seed=3)
    tri, fb, f2t, vb = d.build_faces_host(cells, pos.shape[0])
    assert tri.shape[0] == 12 * n ** 3 + 6 * n ** 2
    assert int(fb.sum()) == 12 * n * n
    P = pos.astype(np.float64)
    vol = np.einsum("ij,ij->i", np.cross(P[cells[:, 1]] - P[cells[:, 0]], P[cells[:, 2]] - P[cells[:, 0]]),
                    P[cells[:, 3]] - P[cells[:, 0]])
    assert (vol < 0).all()  # TetMesh::checkIsAnyTetDegenerate convention


@pytest.mark.parametrize("n", [2, 8])
def test_faces_match_oracle(oracle, n):
    cells, pos = S.kuhn_mesh(n, seed=5)
    tri, fb, f2t, vb = d.build_faces_host(cells, pos.shape[0])
    fa = oracle.Faces(cells, pos.shape[0])
    assert np.array_equal(tri, fa.tri)
    assert np.array_equal(fb, fa.face_boundary)
    assert np.array_equal(f2t, fa.face_to_tet)
    assert np.array_equal(vb, fa.vertex_boundary)


def test_faces_on_unshared_tets(oracle):
    # Two tets sharing one face plus one isolated tet (ragged topology).
    cells = np.array([[0, 1, 2, 3], [1, 0, 2, 4], [5, 6, 7, 8]], np.uint32)
    tri, fb, f2t, vb = d.build_faces_host(cells, 9)
    fa = oracle.Faces(cells, 9)
    assert tri.shape[0] == 11 and int(fb.sum()) == 10
    assert np.array_equal(tri, fa.tri) and np.array_equal(f2t, fa.face_to_tet)


def test_empty_mesh():
    tri, fb, f2t, vb = d.build_faces_host(np.zeros((0, 4), np.uint32), 0)
    assert tri.shape[0] == 0


def test_out_of_range_cell_rejected():
    with pytest.raises(RuntimeError):
        d.build_faces_host(np.array([[0, 1, 2, 9]], np.uint32), 4)


def _remove_transparent_loops(cells, pos, vcol, ccol, thr):
    """removeTransparentTets (TetMesh.cpp:1991-2084) restated with loops."""
    used_v = [False] * pos.shape[0]
    keep = []
    for t, c in enumerate(cells):
        above = any(vcol[v, 3] >= thr for v in c) if vcol is not None else ccol[t, 3] >= thr
        if above:
            keep.append(t)
            for v in c:
                used_v[v] = True
    remap, k = [0] * pos.shape[0], 0
    for v in range(pos.shape[0]):
        remap[v] = k
        k += used_v[v]
    new_cells = np.array([[remap[v] for v in cells[t]] for t in keep], np.uint32).reshape(-1, 4)
    sel = np.array(used_v, bool)
    return (new_cells, pos[sel], None if vcol is None else vcol[sel],
            None if ccol is None else ccol[np.array(keep, np.int64)])


def test_unlink_cells_gives_each_cell_its_own_vertices():
    from difftetvr_b200.tet_mesh import unlink_cells
    cells, pos = S.kuhn_mesh(3, seed=4)
    col = S.gaussian_colors(pos, seed=4)
    c2, p2, v2 = unlink_cells(cells, pos, col)
    assert c2.shape == cells.shape and p2.shape == (4 * cells.shape[0], 3)
    np.testing.assert_array_equal(c2.reshape(-1), np.arange(c2.size))
    np.testing.assert_array_equal(p2[c2], pos[cells])  # every corner in place
    np.testing.assert_array_equal(v2[c2], col[cells])
    tri, fb, _, _ = d.build_faces_host(c2, p2.shape[0])
    assert tri.shape[0] == 4 * cells.shape[0] and fb.all()  # no face shared: all boundary


@pytest.mark.parametrize("per_cell", [False, True])
def test_remove_transparent_cells_matches_loop_restatement(per_cell):
    from difftetvr_b200.tet_mesh import remove_transparent_cells
    rng = np.random.default_rng(11)
    cells, pos = S.kuhn_mesh(4, seed=2)
    vcol = rng.uniform(0, 1, (pos.shape[0], 4)).astype(np.float32)
    vcol[:, 3] = np.where(rng.uniform(size=pos.shape[0]) < 0.8, 0.05, 0.9)
    ccol = rng.uniform(0, 1, (cells.shape[0], 4)).astype(np.float32)
    if per_cell:
        vcol = None
    else:
        ccol = None
    for thr in (0.0, 0.05, 0.5, 2.0):
        got = remove_transparent_cells(cells, pos, vcol, ccol, thr)
        want = _remove_transparent_loops(cells, pos, vcol, ccol, thr)
        for g, w in zip(got, want):
            if w is None:
                assert g is None
            else:
                np.testing.assert_array_equal(g, w)
        if thr == 0.0:
            np.testing.assert_array_equal(got[0], cells)  # nothing removed
        if thr == 0.05 and not per_cell:  # alpha == threshold keeps a cell
            np.testing.assert_array_equal(got[0], cells)
        if thr == 0.5:
            assert 0 < got[0].shape[0] < cells.shape[0]
        if thr == 2.0:
            assert got[0].shape == (0, 4) and got[1].shape == (0, 3)
