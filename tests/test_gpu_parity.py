"""CUDA path vs the CPU oracle (B200).  Fragment lists bit-exact; images within
1e-5 absolute of the FP64 oracle; gradients within 1e-4 relative (norm) of the
FP64 oracle's exact adjoint."""
import numpy as np
import pytest
import torch

from helpers import Scene, rel_err, two_block_scene

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5     # absolute, FP32 image vs FP64 oracle
GRAD_TOL = 1e-4    # relative (L2 norm), FP32 adjoint vs FP64 oracle adjoint


def _oracle_all(O, sc, w=None, ert=None):
    fa = O.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(O)
    prm = sc.oracle_params(O) if ert is None else O.make_params(
        attenuation=sc.attenuation, use_ert=ert, clear=sc.clear)
    img, tf, term, nf = O.render(fa, sc.pos, sc.col, cam, prm)
    out = {"faces": fa, "cam": cam, "prm": prm, "img": img, "tf": tf, "term": term, "nf": nf}
    if w is not None:
        out["gp"], out["gc"] = O.adjoint(fa, sc.pos, sc.col, cam, prm, w)
    return out


# (2, 512): every face's box is over 64 px (64-bit edge functions);
# (1, 3072): boxes of more than 2^21 pixels (row-by-row walk).
@pytest.mark.parametrize("n,res", [(8, 128), (16, 512), (32, 256), (2, 512), (1, 3072)])
def test_fragment_lists_bit_exact(oracle, n, res):
    sc = Scene(n, res, seed=n)
    mesh, r = sc.make_renderer()
    r.render()
    torch.cuda.synchronize()
    off_g, rec_g = r.get_fragment_lists()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    off_o, rec_o = oracle.fragments(fa, sc.pos, sc.oracle_camera(oracle))
    assert np.array_equal(off_g.astype(np.int64), off_o)
    assert rec_g.shape == rec_o.shape
    assert np.array_equal(rec_g, rec_o)
    if (n, res) == (16, 512):
        # Every length of the one-thread class (2..8) and the first of the
        # warp classes (9) occurs here.
        lens = np.diff(off_o)
        assert all((lens == k).any() for k in range(2, 10))


def test_long_lists_bit_exact_and_composited(oracle):
    """A 4 x 4 x 600-cell column seen end-on: per-pixel lists of well over 1024
    fragments (register, shared-memory and block sorts all run)."""
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    cells, pos = d.build_hex_mesh((-0.1, -0.1, -1.0), (0.1, 0.1, 1.0), 5, 5, 601)
    col = S.gaussian_colors(pos, seed=3)
    col[:, 3] *= 0.05
    view = S.look_at_view([0.02, 0.03, 2.5])
    mesh = d.TetMesh()
    mesh.set_use_gradients(True)
    mesh.set_tet_mesh_data(cells, pos, col)
    r = d.Renderer(d.RendererType.PPLL)
    r.set_tet_mesh(mesh)
    r.set_viewport_size(48, 48)
    r.set_camera_fovy(S.FOVY_45)
    r.set_view_matrix(view)
    r.set_attenuation(1.0)
    r.set_use_early_ray_termination(False)
    img = r.render().cpu().numpy().astype(np.float64)
    off_g, rec_g = r.get_fragment_lists()
    fa = oracle.Faces(cells, pos.shape[0])
    cam = oracle.make_camera(view, S.FOVY_45, 48, 48)
    off_o, rec_o = oracle.fragments(fa, pos, cam)
    lens = np.diff(off_o)
    assert lens.max() > 1024 and ((lens > 32) & (lens <= 512)).any() and ((lens > 512) & (lens <= 1024)).any()
    assert np.array_equal(off_g.astype(np.int64), off_o) and np.array_equal(rec_g, rec_o)
    # Every sort method of every list-length class (distribution sorts included).
    for bucket in (0x00, 0x3e):
        for surrogate in (0x00, 0x1e):
            r.set_tuning(sort_bucket_classes=bucket, sort_surrogate_classes=surrogate)
            img_t = r.render().cpu().numpy().astype(np.float64)
            off_t, rec_t = r.get_fragment_lists()
            assert np.array_equal(off_t, off_g) and np.array_equal(rec_t, rec_g), (bucket, surrogate)
            assert np.array_equal(img_t, img)
    img_o = oracle.render(fa, pos, col, cam, oracle.make_params(attenuation=1.0))[0]
    # Thousands of segments per pixel: FP32 accumulation error of the
    # composite grows with the list length; this stress case is held to 1e-4.
    assert np.abs(img - img_o).max() < 1e-4


@pytest.mark.parametrize("cells_z", [6000, 14000])
def test_lists_over_block_cap_bit_exact(oracle, cells_z):
    """A 1 x 1 x N-cell column seen end-on puts about 3 N fragments in the
    centre pixels' lists (18,000 and 42,000: one and two merge stages past
    the 16,384 records a block sorts in shared memory).  Every list is sorted
    bit-exactly and composited."""
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    cells, pos = d.build_hex_mesh((-0.05, -0.05, -1.0), (0.05, 0.05, 1.0), 2, 2, cells_z + 1)
    col = S.gaussian_colors(pos, seed=5)
    col[:, 3] *= 1e-3
    view = S.look_at_view([0.001, 0.002, 2.5])
    mesh = d.TetMesh()
    mesh.set_tet_mesh_data(cells, pos, col)
    r = d.Renderer(d.RendererType.PPLL)
    r.set_tet_mesh(mesh)
    r.set_viewport_size(64, 64)
    r.set_camera_fovy(S.FOVY_45)
    r.set_view_matrix(view)
    r.set_attenuation(1.0)
    r.set_use_early_ray_termination(False)
    img = r.render().cpu().numpy().astype(np.float64)
    off_g, rec_g = r.get_fragment_lists()
    fa = oracle.Faces(cells, pos.shape[0])
    cam = oracle.make_camera(view, S.FOVY_45, 64, 64)
    off_o, rec_o = oracle.fragments(fa, pos, cam)
    assert np.diff(off_o).max() > 16384 * (1 if cells_z < 10000 else 2)
    assert np.array_equal(off_g.astype(np.int64), off_o) and np.array_equal(rec_g, rec_o)
    img_o = oracle.render(fa, pos, col, cam, oracle.make_params(attenuation=1.0))[0]
    assert np.abs(img - img_o).max() < 1e-4  # tens of thousands of FP32 segments per pixel


def test_mesh_faces_match_oracle(oracle):
    sc = Scene(8, 64, seed=3)
    mesh, r = sc.make_renderer()
    tri, fb, f2t, vb = mesh.native.copy_faces()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    assert np.array_equal(tri, fa.tri) and np.array_equal(fb, fa.face_boundary)
    assert np.array_equal(f2t, fa.face_to_tet) and np.array_equal(vb, fa.vertex_boundary)


@pytest.mark.parametrize("n,res,clear", [(8, 128, (0, 0, 0, 0)), (16, 512, (0, 0, 0, 0)),
                                         (8, 96, (0.2, 0.4, 0.6, 0.5))])
def test_image_matches_fp64_oracle(oracle, n, res, clear):
    sc = Scene(n, res, seed=n + 1, clear=clear)
    mesh, r = sc.make_renderer()
    img = r.render().cpu().numpy()
    o = _oracle_all(oracle, sc)
    e = np.abs(img.astype(np.float64) - o["img"]).max(-1)
    y, x = np.unravel_index(int(e.argmax()), e.shape)
    assert e.max() < IMG_TOL, (float(e.max()), (y, x), img[y, x].tolist(), o["img"][y, x].tolist(),
                               int((e > IMG_TOL).sum()))
    assert r.get_num_fragments() == o["nf"]


def test_image_with_early_ray_termination(oracle):
    """ERT on (threshold 1e-4, attenuation 4): the termination index is a discrete
    function of FP32 vs FP64 transmittance, so a pixel whose T lands within
    rounding of the threshold may stop one segment apart; such pixels differ by
    at most T * (segment opacity) <= thresh."""
    sc = Scene(16, 256, seed=9, attenuation=4.0, ert=True)
    mesh, r = sc.make_renderer()
    img = r.render().cpu().numpy().astype(np.float64)
    tf_g, term_g = r.get_pixel_state()
    o = _oracle_all(oracle, sc)
    same = term_g == o["term"]
    assert same.mean() > 0.999
    err = np.abs(img - o["img"]).max(-1)
    assert err[same].max() < IMG_TOL
    assert err.max() < 1e-4
    assert (term_g < np.diff(r.get_fragment_lists()[0]).reshape(256, 256)).sum() > 100  # ERT actually fired


# two_blocks: rays leave one block and enter the other, so consecutive faces of
# a list share no vertex there (every cached vertex row is written out).
# (16, 512): the 16^3 / 512^2 configuration the reference runs on the CPU,
# with and without early ray termination.
@pytest.mark.parametrize("kind,n,res,ert", [("cube", 8, 128, False), ("cube", 16, 256, False),
                                            ("cube", 8, 128, True), ("two_blocks", 4, 128, False),
                                            ("cube", 16, 512, False), ("cube", 16, 512, True)])
def test_gradients_match_fp64_oracle(oracle, kind, n, res, ert):
    if kind == "two_blocks":
        sc = two_block_scene(n, res, seed=20 + n)
    else:
        sc = Scene(n, res, seed=20 + n, attenuation=2.0 if ert else 1.0, ert=ert)
    mesh, r = sc.make_renderer()
    rng = np.random.default_rng(5)
    w = rng.normal(size=(res, res, 4)).astype(np.float32)
    img = r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda())
    gp = pos.grad.cpu().numpy()
    gc = col.grad.cpu().numpy()
    o = _oracle_all(oracle, sc, w=w.astype(np.float64))
    if ert:
        _, term_g = r.get_pixel_state()
        assert (term_g == o["term"]).mean() > 0.999
    assert rel_err(gp, o["gp"]) < GRAD_TOL, rel_err(gp, o["gp"])
    assert rel_err(gc, o["gc"]) < GRAD_TOL, rel_err(gc, o["gc"])


@pytest.mark.parametrize("kind,n,res", [("cube", 8, 128), ("cube", 16, 256), ("two_blocks", 4, 128)])
def test_absolute_gradients_match_fp64_oracle(oracle, kind, n, res):
    """render_adjoint(use_abs_grad=True): per fragment and vertex, the absolute
    value of each position and colour contribution (Backward.glsl:449-468),
    summed over the fragments; world-space rows through the id-searched
    vertex cache."""
    sc = two_block_scene(n, res, seed=40 + n) if kind == "two_blocks" else Scene(n, res, seed=40 + n)
    mesh, r = sc.make_renderer()
    w = np.random.default_rng(6).normal(size=(res, res, 4)).astype(np.float32)
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda(), use_abs_grad=True)
    gp, gc = pos.grad.cpu().numpy(), col.grad.cpu().numpy()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    gp_o, gc_o = oracle.adjoint(fa, sc.pos, sc.col, sc.oracle_camera(oracle), sc.oracle_params(oracle, use_abs_grad=True),
                                w.astype(np.float64))
    assert (gc >= 0).all() and rel_err(gp, gp_o) < GRAD_TOL and rel_err(gc, gc_o) < GRAD_TOL, \
        (rel_err(gp, gp_o), rel_err(gc, gc_o))


def test_gradients_vs_fp64_central_differences(oracle):
    """CUDA adjoint vs FP64 central differences (step 1e-4, Richardson-refined)
    of the forward with frozen fragment lists: 64 position coordinates + 64
    RGBA values of an 8^3 mesh at 128^2."""
    from test_oracle import _fd_pairs
    sc = Scene(8, 128, seed=11)
    mesh, r = sc.make_renderer()
    rng = np.random.default_rng(11)
    w = rng.normal(size=(128, 128, 4))
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w.astype(np.float32)).cuda())
    gp = pos.grad.cpu().numpy().astype(np.float64)
    gc = col.grad.cpu().numpy().astype(np.float64)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)
    loss = lambda p, c: float((oracle.render_frozen(fa, sc.pos, p, c, cam, prm) * w).sum())  # noqa: E731
    fd, an, rel = _fd_pairs(oracle, loss, gp, gc, sc.pos.astype(np.float64), sc.col.astype(np.float64),
                            np.random.default_rng(3), richardson=True)
    assert np.median(rel) < 1e-5
    assert rel.max() < 1e-3, np.sort(rel)[-5:]
    assert rel_err(fd, an) < 1e-4


def test_deterministic_lists_and_images():
    sc = Scene(16, 256, seed=2)
    mesh, r = sc.make_renderer()
    a = r.render().clone()
    la = r.get_fragment_lists()
    b = r.render().clone()
    lb = r.get_fragment_lists()
    assert torch.equal(a, b)
    assert np.array_equal(la[0], lb[0]) and np.array_equal(la[1], lb[1])


def test_empty_view_and_tiny_viewports(oracle):
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    sc = Scene(4, 32, seed=1)
    mesh, r = sc.make_renderer()
    # Camera looking away from the mesh: no fragments, image = clear colour.
    # Camera at (0, 0, 3) looking along +z, away from the mesh (rotation of 180
    # degrees about y): every vertex lies behind it.
    r.set_view_matrix([-1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1, 0, 0, 0, 3, 1])
    r.set_clear_color(d.vec4(0.25, 0.5, 0.75, 1.0))
    img = r.render()
    assert r.get_num_fragments() == 0
    assert torch.allclose(img, torch.tensor([0.25, 0.5, 0.75, 1.0], device=img.device).expand_as(img))
    # 1x1 and non-square viewports agree with the oracle.
    for (w, h) in [(1, 1), (37, 5), (5, 61)]:
        sc2 = Scene(4, 1, seed=4)
        mesh2, r2 = sc2.make_renderer()
        r2.set_viewport_size(w, h)
        img2 = r2.render().cpu().numpy().astype(np.float64)
        fa = oracle.Faces(sc2.cells, sc2.pos.shape[0])
        cam = oracle.make_camera(sc2.view, sc2.fovy, w, h)
        o = oracle.render(fa, sc2.pos, sc2.col, cam, sc2.oracle_params(oracle))[0]
        assert np.abs(img2 - o).max() < IMG_TOL


def test_budget_error_is_reported():
    from difftetvr_b200._lib import DTV_ERR_BUDGET, DtvError
    sc = Scene(8, 128, seed=1)
    mesh, r = sc.make_renderer()
    r.set_fragment_budget_bytes(1024, over_budget="error")
    with pytest.raises(DtvError) as e:
        r.render()
    assert e.value.code == DTV_ERR_BUDGET
    r.set_fragment_budget_bytes(0)
    r.render()  # recovers: counters were reset
    assert r.get_num_fragments() > 0


def test_render_adjoint_argument_checks():
    sc = Scene(4, 32, seed=1)
    mesh, r = sc.make_renderer()
    r.render()
    with pytest.raises(RuntimeError):
        r.render_adjoint(torch.zeros(32, 32, 3, device="cuda"))
    with pytest.raises(RuntimeError):
        r.render_adjoint(torch.zeros(32, 32, 4, device="cuda", dtype=torch.float64))
    with pytest.raises(RuntimeError):
        r.render_adjoint(torch.zeros(32, 32, 4))


@pytest.mark.parametrize("delta,slivers", [(2e-5, 0), (5e-5, 200), (3e-4, 400)])
def test_edge_on_faces_match_fp64_oracle(oracle, delta, slivers):
    """Faces seen (almost) edge-on: an unjittered 16^3 grid whose planes x = 0
    and y = 0 pass `delta` from the camera centre, so the faces in them project
    to slivers about 1e-4 .. 1e-3 px wide along the centre row and column
    (257 x 257: pixel centres lie on both; at delta = 2e-5 the snapped slivers
    have zero area and only their neighbours graze the centre lines).
    Barycentrics there are ill-conditioned in plain FP32 screen coordinates
    (the oracle's FP32 port is 0.07 off at delta = 2e-5); the
    snapped-plus-residual edge functions keep the image within 1e-5 and the
    gradients within 1e-4 of the FP64 oracle."""
    import difftetvr_b200 as d
    from difftetvr_b200 import synthetic as S
    from helpers import Scene
    sc = Scene(16, 257, seed=13, jitter=0.0)
    sc.view = S.look_at_view([delta, 0.7 * delta, 2.9])
    mesh, r = sc.make_renderer()
    img = r.render().cpu().numpy().astype(np.float64)
    o = _oracle_all(oracle, sc, w=np.random.default_rng(13).normal(size=(257, 257, 4)))
    # Slivers of the two planes really are in the lists along the centre lines.
    off, rec = r.get_fragment_lists()
    faces = (rec & np.uint64(0xFFFFFFFF)) >> np.uint64(2)
    fa = o["faces"]
    tri_pos = sc.pos[fa.tri[faces.astype(np.int64)]]
    in_plane = (np.abs(tri_pos[..., 0]).max(-1) == 0) | (np.abs(tri_pos[..., 1]).max(-1) == 0)
    assert in_plane.sum() >= slivers
    e = np.abs(img - o["img"]).max()
    assert e < IMG_TOL, e
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    w = np.random.default_rng(13).normal(size=(257, 257, 4))
    r.render_adjoint(torch.from_numpy(w.astype(np.float32)).cuda())
    gp = pos.grad.cpu().numpy()
    gc = col.grad.cpu().numpy()
    assert rel_err(gp, o["gp"]) < GRAD_TOL, rel_err(gp, o["gp"])
    assert rel_err(gc, o["gc"]) < GRAD_TOL, rel_err(gc, o["gc"])
