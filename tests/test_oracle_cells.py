"""Pinning the oracle's per-cell colour path (ColorStorage.PER_CELL) on the
CPU: with one colour everywhere it equals the per-vertex path (whose constant-
colour sub-segments compose to the same exp(-a t)); FP64 central differences
of its own forward check the adjoint (positions and cell colours)."""
import numpy as np
import pytest

from difftetvr_b200 import synthetic as S
from helpers import Scene, two_block_scene
from test_oracle import _fd_pairs


@pytest.mark.parametrize("two_blocks,ert", [(False, False), (True, False), (False, True)])
def test_constant_colour_equals_per_vertex_path(oracle, two_blocks, ert):
    sc = two_block_scene(4, 64, seed=3, ert=ert) if two_blocks else Scene(6, 64, seed=5, ert=ert)
    c = np.array([0.3, 0.7, 0.2, 1.7], np.float32)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    prm = oracle.make_params(attenuation=2.0, use_ert=ert, ert_thresh=0.05)
    vcol = np.tile(c, (sc.pos.shape[0], 1))
    ccol = np.tile(c, (sc.cells.shape[0], 1))
    img_v, tf_v, term_v, nf_v = oracle.render(fa, sc.pos, vcol, cam, prm)
    img_c, tf_c, term_c, nf_c = oracle.render_cells(fa, sc.pos, ccol, cam, prm)
    assert nf_c == nf_v and img_c[..., 3].max() > 0.3
    # Where a ray crosses an edge, two consecutive fragments can lie on faces
    # with no common tet: the per-cell rule (tetIdUnion) skips that stretch,
    # the per-vertex path composites it.  Elsewhere both integrate the same
    # segments (across empty space neither does).
    off, rec = oracle.fragments(fa, sc.pos, cam)
    f2t = fa.face_to_tet
    faces = (rec & np.uint64(0xffffffff)).astype(np.int64) >> 2
    bound = ((rec >> np.uint64(1)) & np.uint64(1)).astype(bool)
    front = (rec & np.uint64(1)).astype(bool)
    clean = np.ones(64 * 64, bool)
    for p in range(64 * 64):
        fs = faces[off[p]:off[p + 1]]
        for j in range(1, fs.size):
            a, b = f2t[fs[j - 1]], f2t[fs[j]]
            shared = (a[0] in b and a[0] != 0xffffffff) or (a[1] in b and a[1] != 0xffffffff)
            gap = bound[off[p] + j - 1] and not front[off[p] + j - 1] and bound[off[p] + j] and front[off[p] + j]
            if not shared and not gap:
                clean[p] = False
                break
    clean = clean.reshape(64, 64)
    assert clean.mean() > 0.99
    np.testing.assert_allclose(img_c[clean], img_v[clean], rtol=0, atol=1e-12)
    np.testing.assert_allclose(tf_c[clean], tf_v[clean], rtol=0, atol=1e-12)
    covered = (np.diff(off).reshape(64, 64) > 0) & clean
    if ert:
        # The per-vertex loop counts segments from fragment 1, the per-cell loop
        # fragments from 0: both stop before the same segment.
        assert np.array_equal(term_c[covered], term_v[covered])
        assert (term_c[covered] < np.diff(oracle.fragments(fa, sc.pos, cam)[0]).reshape(64, 64)[covered]).any()


def test_distinct_cell_colours_change_the_image(oracle):
    sc = Scene(4, 48, seed=2)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), oracle.make_params(attenuation=1.0)
    rng = np.random.default_rng(0)
    ccol = rng.uniform(0.1, 3.0, size=(sc.cells.shape[0], 4))
    img1 = oracle.render_cells(fa, sc.pos, ccol, cam, prm)[0]
    ccol2 = ccol.copy()
    ccol2[:, :3] = ccol[:, :3][::-1]
    img2 = oracle.render_cells(fa, sc.pos, ccol2, cam, prm)[0]
    assert np.abs(img1 - img2).max() > 1e-2


@pytest.mark.parametrize("ert", [False, True])
def test_adjoint_matches_central_differences(oracle, ert):
    sc = Scene(6, 64, seed=9, ert=ert)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam = sc.oracle_camera(oracle)
    prm = oracle.make_params(attenuation=3.0, use_ert=ert, ert_thresh=0.02)
    rng = np.random.default_rng(1)
    ccol = rng.uniform(0.2, 2.5, size=(sc.cells.shape[0], 4))
    w = rng.normal(size=(64, 64, 4))
    pos = sc.pos.astype(np.float64)
    _, _, term, _, gp, gc = oracle.render_cells(fa, pos, ccol, cam, prm, image_adjoint=w)
    if ert:
        lens = np.diff(oracle.fragments(fa, sc.pos, cam)[0]).reshape(64, 64)
        assert (term < lens).sum() > 20

    def loss(p, c):
        return float((oracle.render_cells(fa, p, c, cam, prm, positions_coverage=sc.pos)[0] * w).sum())

    # Position coordinates: central differences at steps h and h/2; a
    # coordinate whose two differences disagree sits on a discontinuity (a
    # face turning edge-on at some pixel flips its barycentric weights) and is
    # left out.
    cand = np.flatnonzero(np.abs(gp).sum(1) > 0)
    fd, an = [], []
    h = 1e-4
    for k in np.random.default_rng(3).choice(cand.size * 3, size=48, replace=False):
        idx = (cand[k // 3], k % 3)

        def cd(step):
            xp, xm = pos.copy(), pos.copy()
            xp[idx] += step
            xm[idx] -= step
            return (loss(xp, ccol) - loss(xm, ccol)) / (2 * step)

        d1, d2 = cd(h), cd(h / 2)
        if abs(d1 - d2) > 1e-3 * max(abs(d2), 1.0):
            continue
        fd.append((4 * d2 - d1) / 3)
        an.append(gp[idx])
    fd, an = np.array(fd), np.array(an)
    assert fd.size >= (32 if ert else 44)  # ERT: the termination index jumps too
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-4
    cand = np.flatnonzero(np.abs(gc).sum(1) > 0)
    out = []
    for k in np.random.default_rng(4).choice(cand.size * 4, size=48, replace=False):
        idx = (cand[k // 4], k % 4)
        cp, cm = ccol.copy(), ccol.copy()
        cp[idx] += 1e-5
        cm[idx] -= 1e-5
        out.append(((loss(pos, cp) - loss(pos, cm)) / 2e-5, gc[idx]))
    fd, an = np.array(out).T
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-6
