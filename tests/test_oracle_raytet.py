"""Pinning the oracle's ray-tet (intersection) path on the CPU: closed form on
one tet with the Euclidean chord, segment counts on convex meshes, equality
with the fragment-list path where both define the same integral, and FP64
central differences of its own forward."""
import numpy as np
import pytest

from difftetvr_b200 import synthetic as S
from helpers import Scene, two_block_scene
from test_oracle import _fd_pairs, analytic_single_tet_depths


def _ray_scale(W, H, fovy):
    f = 0.5 * H / np.tan(0.5 * float(np.float32(fovy)))
    xs = (np.arange(W) + 0.5 - 0.5 * W) / f
    ys = (np.arange(H) + 0.5 - 0.5 * H) / f
    return np.sqrt(1.0 + xs[None, :] ** 2 + ys[:, None] ** 2)


def test_single_tet_closed_form_euclidean_chord(oracle):
    """Constant colour c and density a: image = (1 - exp(-a L)) (c, 1) with L the
    Euclidean chord of the pixel ray through the tet
    (IntersectRasterization.glsl:139-273 integrates along the normalised ray)."""
    pos = np.array([[-0.1, -0.1, 0.1], [0.1, -0.1, 0.1], [0.0, 0.3, 0.0], [0.1, -0.1, -0.1]], np.float32) * 4.0
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    c, a = np.array([0.3, 0.6, 0.9]), 2.5
    col = np.tile(np.r_[c, a].astype(np.float32), (4, 1))
    W = H = 48
    view = S.look_at_view([0.7, 0.9, 2.6])
    fa = oracle.Faces(cells, 4)
    img, tf, nseg = oracle.raytet(fa, pos, col, oracle.make_camera(view, S.FOVY_45, W, H),
                                  oracle.make_params(attenuation=1.0))
    z = analytic_single_tet_depths(pos, view, S.FOVY_45, W, H)
    hit = ~np.isnan(z[..., 0])
    L = np.where(hit, (z[..., 1] - z[..., 0]) * _ray_scale(W, H, S.FOVY_45), 0.0)
    alpha = 1.0 - np.exp(-a * L)
    c32 = c.astype(np.float32).astype(np.float64)
    expect = np.concatenate([alpha[..., None] * c32, alpha[..., None]], -1)
    err = np.abs(img - expect).max(-1)
    assert hit.sum() > 100
    assert np.quantile(err, 0.99) < 1e-9
    assert err.max() < 2e-3
    assert set(np.unique(nseg)) <= {0, 1} and (nseg == 1).sum() > 100


@pytest.mark.parametrize("n,res,seed", [(4, 64, 1), (8, 96, 5)])
def test_segments_equal_fragments_minus_one_on_convex_mesh(oracle, n, res, seed):
    """A pixel ray through the convex jittered cube crosses k tets and k + 1
    faces, so the walk composites exactly (list length - 1) segments."""
    sc = Scene(n, res, seed=seed)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    off, _ = oracle.fragments(fa, sc.pos, cam)
    lens = np.diff(off).reshape(res, res)
    _, _, nseg = oracle.raytet(fa, sc.pos, sc.col, cam, sc.oracle_params(oracle))
    covered = lens > 0
    assert covered.sum() > 0.2 * res * res
    np.testing.assert_array_equal(nseg[covered], lens[covered] - 1)
    assert np.all(nseg[~covered] == 0)


@pytest.mark.parametrize("two_blocks", [False, True])
def test_matches_fragment_list_path_on_the_optical_axis(oracle, two_blocks):
    """At the centre pixel of a 1 x 1 viewport the ray runs along the optical
    axis (chord = view-depth difference), so the ray-tet walk and the
    fragment-list composite integrate the same segments: the images agree to
    FP64 rounding, also across an empty gap between two meshes."""
    sc = two_block_scene(3, 1, seed=2) if two_blocks else Scene(6, 1, seed=3)
    if not two_blocks:
        sc.view = S.look_at_view([0.31, 0.42, 2.7])
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = oracle.make_camera(sc.view, sc.fovy, 1, 1)
    prm = oracle.make_params(attenuation=1.5)
    off, rec = oracle.fragments(fa, sc.pos, cam)
    assert off[-1] >= (8 if two_blocks else 4)
    bound = ((rec >> np.uint64(1)) & np.uint64(1)).sum()
    assert bound == (4 if two_blocks else 2)
    img_l = oracle.render(fa, sc.pos, sc.col, cam, prm)[0]
    img_r, _, nseg = oracle.raytet(fa, sc.pos, sc.col, cam, prm)
    assert int(nseg[0, 0]) == int(off[-1]) - (2 if two_blocks else 1)
    np.testing.assert_allclose(img_r, img_l, rtol=0, atol=1e-12)


@pytest.mark.parametrize("two_blocks", [False, True])
def test_adjoint_matches_fp64_central_differences(oracle, two_blocks):
    """FP64 analytic adjoint of the walk vs Richardson-refined central
    differences (step 1e-4) of the forward with frozen coverage: 64 position
    coordinates + 64 RGBA values."""
    sc = two_block_scene(3, 64, seed=4) if two_blocks else Scene(6, 64, seed=7)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)
    rng = np.random.default_rng(17)
    w = rng.normal(size=(64, 64, 4))
    pos64, col64 = sc.pos.astype(np.float64), sc.col.astype(np.float64)
    _, _, nseg, gp, gc = oracle.raytet(fa, pos64, col64, cam, prm, image_adjoint=w)
    if two_blocks:
        off, rec = oracle.fragments(fa, sc.pos, cam)
        bound = np.add.reduceat(((rec >> np.uint64(1)) & np.uint64(1)).astype(np.int64),
                                off[:-1][np.diff(off) > 0])
        assert (bound == 4).sum() > 50  # rays that cross both meshes

    def loss(p, c):
        img = oracle.raytet(fa, p, c, cam, prm, positions_coverage=sc.pos)[0]
        return float((img * w).sum())

    fd, an, rel = _fd_pairs(oracle, loss, gp, gc, pos64, col64, np.random.default_rng(3), richardson=True)
    assert np.median(rel) < 1e-5
    assert rel.max() < 1e-3, np.sort(rel)[-5:]
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-4
