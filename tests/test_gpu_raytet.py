"""CUDA ray-tet (intersection renderer) path vs the CPU oracle (B200).
Boundary fragment lists bit-exact; per-pixel segment counts exact; images
within 1e-5 absolute of the FP64 oracle; gradients within 1e-4 relative (norm)
of the FP64 oracle's adjoint and of FP64 central differences."""
import numpy as np
import pytest
import torch

from helpers import Scene, rel_err, two_block_scene

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_TOL = 1e-4


def _intersection():
    import difftetvr_b200 as d
    return d.RendererType.INTERSECTION


def _scene(kind, n, res, seed, **kw):
    return two_block_scene(n, res, seed=seed, **kw) if kind == "two_blocks" else Scene(n, res, seed=seed, **kw)


@pytest.mark.parametrize("kind,n,res", [("cube", 8, 128), ("cube", 16, 256), ("two_blocks", 4, 128)])
def test_boundary_lists_bit_exact(oracle, kind, n, res):
    sc = _scene(kind, n, res, seed=n + 2)
    mesh, r = sc.make_renderer(_intersection())
    r.render()
    torch.cuda.synchronize()
    off_g, rec_g = r.get_fragment_lists()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    off_o, rec_o = oracle.fragments(fa, sc.pos, sc.oracle_camera(oracle))
    keep = ((rec_o >> np.uint64(1)) & np.uint64(1)) == 1
    pix = np.repeat(np.arange(res * res), np.diff(off_o))
    off_b = np.zeros(res * res + 1, np.int64)
    np.cumsum(np.bincount(pix[keep], minlength=res * res), out=off_b[1:])
    assert np.array_equal(off_g.astype(np.int64), off_b)
    assert np.array_equal(rec_g, rec_o[keep])


def test_inconsistently_oriented_tets_walk_like_the_oracle(oracle):
    """Every other tet stored with two vertices swapped, so neighbouring tets
    list their shared faces with the same winding.  The walk classifies a
    tet's faces by the stored winding and the owner rule, which assume
    consistently oriented tets (here most walks stop after a tet or two); the
    per-tet classification bits must reproduce the oracle's rule exactly,
    segment for segment."""
    sc = Scene(6, 96, seed=9)
    cells = sc.cells.copy()
    cells[::2, [1, 2]] = cells[::2, [2, 1]]
    sc.cells = cells
    mesh, r = sc.make_renderer(_intersection())
    img = r.render().cpu().numpy().astype(np.float64)
    _, nseg_g = r.get_pixel_state()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    img_o, _, nseg_o = oracle.raytet(fa, sc.pos, sc.col, sc.oracle_camera(oracle), sc.oracle_params(oracle))
    assert np.array_equal(nseg_g, nseg_o)
    assert (nseg_o > 0).sum() > 0.1 * 96 * 96
    # Walks through mis-oriented tets take segments of negative length, so T
    # grows above 1 (to about 7) and pixel values reach -6: the FP32 depth
    # difference of a segment carries ~2^-24 |z| of error into the optical
    # depth, scaled by T.  The image tolerance is taken relative to the value.
    assert (np.abs(img - img_o) / np.maximum(1.0, np.abs(img_o))).max() < IMG_TOL


@pytest.mark.parametrize("kind,n,res,clear", [("cube", 8, 128, (0, 0, 0, 0)), ("cube", 16, 256, (0, 0, 0, 0)),
                                              ("cube", 8, 96, (0.2, 0.4, 0.6, 0.5)),
                                              ("two_blocks", 4, 128, (0, 0, 0, 0))])
def test_image_and_segments_match_fp64_oracle(oracle, kind, n, res, clear):
    sc = _scene(kind, n, res, seed=n + 1)
    sc.clear = clear
    mesh, r = sc.make_renderer(_intersection())
    img = r.render().cpu().numpy().astype(np.float64)
    tf_g, nseg_g = r.get_pixel_state()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    img_o, tf_o, nseg_o = oracle.raytet(fa, sc.pos, sc.col, sc.oracle_camera(oracle), sc.oracle_params(oracle))
    assert np.array_equal(nseg_g, nseg_o)
    assert (nseg_o > 0).sum() > 0.1 * res * res
    e = np.abs(img - img_o).max(-1)
    y, x = np.unravel_index(int(e.argmax()), e.shape)
    assert e.max() < IMG_TOL, (float(e.max()), (y, x), int((e > IMG_TOL).sum()))


def test_image_with_early_ray_termination(oracle):
    """ERT (threshold 1e-4, attenuation 4) stops the walk before the first tet
    entered with T below the threshold; pixels whose FP32 and FP64 T straddle
    the threshold may stop one tet apart, differing by at most the threshold."""
    sc = Scene(16, 256, seed=9, attenuation=4.0, ert=True)
    mesh, r = sc.make_renderer(_intersection())
    img = r.render().cpu().numpy().astype(np.float64)
    _, nseg_g = r.get_pixel_state()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    img_o, _, nseg_o = oracle.raytet(fa, sc.pos, sc.col, cam, sc.oracle_params(oracle))
    _, _, nseg_full = oracle.raytet(fa, sc.pos, sc.col, cam, oracle.make_params(attenuation=4.0))
    same = nseg_g == nseg_o
    assert same.mean() > 0.999
    err = np.abs(img - img_o).max(-1)
    assert err[same].max() < IMG_TOL
    assert err.max() < 1e-4
    assert (nseg_o < nseg_full).sum() > 100  # ERT actually fired


# (16, 512): the 16^3 / 512^2 configuration the reference runs on the CPU.
@pytest.mark.parametrize("kind,n,res,ert", [("cube", 8, 128, False), ("cube", 16, 256, False),
                                            ("cube", 8, 128, True), ("two_blocks", 4, 128, False),
                                            ("cube", 16, 512, False), ("cube", 16, 512, True)])
def test_gradients_match_fp64_oracle(oracle, kind, n, res, ert):
    sc = _scene(kind, n, res, seed=20 + n, attenuation=2.0 if ert else 1.0, ert=ert)
    mesh, r = sc.make_renderer(_intersection())
    w = np.random.default_rng(5).normal(size=(res, res, 4)).astype(np.float32)
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda())
    gp, gc = pos.grad.cpu().numpy(), col.grad.cpu().numpy()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    _, _, nseg_o, gp_o, gc_o = oracle.raytet(fa, sc.pos.astype(np.float64), sc.col.astype(np.float64),
                                             sc.oracle_camera(oracle), sc.oracle_params(oracle),
                                             image_adjoint=w.astype(np.float64))
    if ert:
        assert (r.get_pixel_state()[1] == nseg_o).mean() > 0.999
    assert rel_err(gp, gp_o) < GRAD_TOL, rel_err(gp, gp_o)
    assert rel_err(gc, gc_o) < GRAD_TOL, rel_err(gc, gc_o)


@pytest.mark.parametrize("kind,n,res", [("cube", 8, 128), ("two_blocks", 4, 128)])
def test_absolute_gradients_match_fp64_oracle(oracle, kind, n, res):
    """render_adjoint(use_abs_grad=True) on the walk: absolute value of each
    fragment's contribution per vertex (world-space rows, straight atomics)."""
    sc = _scene(kind, n, res, seed=40 + n)
    mesh, r = sc.make_renderer(_intersection())
    w = np.random.default_rng(6).normal(size=(res, res, 4)).astype(np.float32)
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w).cuda(), use_abs_grad=True)
    gp, gc = pos.grad.cpu().numpy(), col.grad.cpu().numpy()
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    _, _, _, gp_o, gc_o = oracle.raytet(fa, sc.pos.astype(np.float64), sc.col.astype(np.float64),
                                        sc.oracle_camera(oracle), sc.oracle_params(oracle, use_abs_grad=True),
                                        image_adjoint=w.astype(np.float64))
    assert (gc >= 0).all() and rel_err(gp, gp_o) < GRAD_TOL and rel_err(gc, gc_o) < GRAD_TOL, \
        (rel_err(gp, gp_o), rel_err(gc, gc_o))


def test_gradients_vs_fp64_central_differences(oracle):
    """CUDA ray-tet adjoint vs FP64 central differences (step 1e-4,
    Richardson-refined) of the oracle's forward with frozen coverage: 64
    position coordinates + 64 RGBA values of an 8^3 mesh at 128^2."""
    from test_oracle import _fd_pairs
    sc = Scene(8, 128, seed=11)
    mesh, r = sc.make_renderer(_intersection())
    w = np.random.default_rng(11).normal(size=(128, 128, 4))
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(torch.from_numpy(w.astype(np.float32)).cuda())
    gp = pos.grad.cpu().numpy().astype(np.float64)
    gc = col.grad.cpu().numpy().astype(np.float64)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)

    def loss(p, c):
        return float((oracle.raytet(fa, p, c, cam, prm, positions_coverage=sc.pos)[0] * w).sum())

    fd, an, rel = _fd_pairs(oracle, loss, gp, gc, sc.pos.astype(np.float64), sc.col.astype(np.float64),
                            np.random.default_rng(3), richardson=True)
    assert np.median(rel) < 1e-5
    assert rel.max() < 1e-3, np.sort(rel)[-5:]
    assert rel_err(fd, an) < 1e-4


@pytest.mark.parametrize("ray_tet", [False, True])
def test_render_adjoint_into_equals_render_adjoint(ray_tet):
    import difftetvr_b200 as d
    sc = Scene(8, 96, seed=6)
    mesh, r = sc.make_renderer(_intersection() if ray_tet else d.RendererType.PPLL)
    w = torch.randn(96, 96, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    r.render()
    pos, col = mesh.get_vertex_positions(), mesh.get_vertex_colors()
    pos.grad.zero_()
    col.grad.zero_()
    r.render_adjoint(w)
    gp = torch.zeros_like(pos.detach())
    gc = torch.zeros_like(col.detach())
    r.render_adjoint_into(w, gp, gc)
    torch.cuda.synchronize()
    # Float atomics accumulate in arrival order: equal up to summation order.
    assert rel_err(gp.cpu().numpy(), pos.grad.cpu().numpy()) < 1e-6
    assert rel_err(gc.cpu().numpy(), col.grad.cpu().numpy()) < 1e-6
    with pytest.raises(RuntimeError):
        r.render_adjoint_into(w, gp[:, :2].contiguous(), gc)


def test_walk_is_deterministic_and_differs_from_list_path_off_axis():
    """Same inputs give bitwise-equal images; off the optical axis the ray-tet
    chord is longer than the view-depth difference, so it is more opaque."""
    import difftetvr_b200 as d
    sc = Scene(8, 128, seed=3)
    _, r = sc.make_renderer(_intersection())
    a = r.render().clone()
    b = r.render().clone()
    assert torch.equal(a, b)
    _, rl = sc.make_renderer(d.RendererType.PPLL)
    c = rl.render()
    covered = c[..., 3] > 1e-3
    assert bool((a[..., 3][covered] >= c[..., 3][covered] - 1e-6).all())
