"""Topology edits of TetMesh (unlink_tets, remove_transparent_tets;
TetMesh.cpp:1950-2084) followed by renders on the B200 against the CPU oracle
on the edited arrays: lists bit-exact, images within 1e-5, gradients within
1e-4 relative."""
import numpy as np
import pytest
import torch

from helpers import Scene, rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_TOL = 1e-4


def _check_against_oracle(oracle, mesh, r, sc):
    cells = mesh.get_cells()
    pos = mesh.get_vertex_positions().detach().cpu().numpy()
    col = mesh.get_vertex_colors().detach().cpu().numpy()
    res = sc.res
    w = np.random.default_rng(9).normal(size=(res, res, 4)).astype(np.float32)
    img = r.render().cpu().numpy().astype(np.float64)
    off_g, rec_g = r.get_fragment_lists()
    mesh.get_vertex_positions().grad.zero_()
    mesh.get_vertex_colors().grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda())
    gp = mesh.get_vertex_positions().grad.cpu().numpy()
    gc = mesh.get_vertex_colors().grad.cpu().numpy()
    fa = oracle.Faces(cells, pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)
    off_o, rec_o = oracle.fragments(fa, pos, cam)
    assert np.array_equal(off_g.astype(np.int64), off_o) and np.array_equal(rec_g, rec_o)
    img_o = oracle.render(fa, pos, col, cam, prm)[0]
    assert np.abs(img - img_o).max() < IMG_TOL
    gp_o, gc_o = oracle.adjoint(fa, pos, col, cam, prm, w.astype(np.float64))
    assert rel_err(gp, gp_o) < GRAD_TOL and rel_err(gc, gc_o) < GRAD_TOL, (rel_err(gp, gp_o), rel_err(gc, gc_o))
    return img, rec_g


def test_unlinked_mesh_matches_oracle(oracle):
    """Every cell with its own vertices: no face is shared, so each interior
    face of the original mesh gives two coincident boundary fragments (equal
    depth keys, ordered by face index)."""
    sc = Scene(6, 128, seed=61)
    mesh, r = sc.make_renderer()
    n_cells = mesh.get_num_cells()
    mesh.unlink_tets()
    r.set_tet_mesh(mesh)
    assert mesh.get_num_cells() == n_cells and mesh.get_num_vertices() == 4 * n_cells
    assert mesh.get_num_faces() == 4 * n_cells
    _, rec = _check_against_oracle(oracle, mesh, r, sc)
    depth = (rec >> np.uint64(32)).astype(np.uint32)
    assert (depth[1:] == depth[:-1]).sum() > 1000  # coincident fragments met


def test_remove_transparent_tets_matches_oracle(oracle):
    sc = Scene(8, 128, seed=62)
    rng = np.random.default_rng(62)
    sc.col[:, 3] = np.where(rng.uniform(size=sc.pos.shape[0]) < 0.7, 0.01, 0.8).astype(np.float32)
    mesh, r = sc.make_renderer()
    from difftetvr_b200.tet_mesh import remove_transparent_cells
    want_cells, want_pos, _, _ = remove_transparent_cells(sc.cells, sc.pos, sc.col, None, 0.5)
    mesh.remove_transparent_tets(0.5)
    r.set_tet_mesh(mesh)
    assert 0 < mesh.get_num_cells() < sc.cells.shape[0]
    np.testing.assert_array_equal(mesh.get_cells(), want_cells)
    np.testing.assert_array_equal(mesh.get_vertex_positions().detach().cpu().numpy(), want_pos)
    assert (mesh.get_vertex_colors().detach().cpu().numpy()[mesh.get_cells(), 3] >= 0.5).any(axis=1).all()
    _check_against_oracle(oracle, mesh, r, sc)
