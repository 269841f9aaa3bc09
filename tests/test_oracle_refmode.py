"""The oracle's reference mode: the reference's own formulas of the PPLL path
(NDC depth stored in FP32 and re-linearised, unsigned world-space barycentrics,
the a < 1e-6 drop; the adjoint that skips sub-segment 0, differentiates the
Euclidean segment length and holds the world point fixed), restated from the
GLSL the oracle cites.  These tests pin the restatement where the reference's
own mathematics allows it and record how far it is from the exact path."""
import numpy as np
import pytest

from helpers import Scene, rel_err


def test_bary_adjoint_is_the_derivative_of_the_unsigned_weights(oracle):
    """baryAdjoint (BackwardCommon.glsl:183-251) is the derivative of the
    unsigned weights u, v with the world point held fixed: FP64 central
    differences of u and v over the nine vertex coordinates."""
    rng = np.random.default_rng(1)
    for _ in range(20):
        p0, p1, p2 = rng.normal(size=(3, 3))
        lam = rng.uniform(0.05, 0.9, 3)
        lam /= lam.sum()
        p = lam[0] * p0 + lam[1] * p1 + lam[2] * p2 + 1e-3 * rng.normal(size=3)
        u, v, du, dv = oracle.refmode_bary_uv(p, p0, p1, p2)
        h = 1e-6
        for j in range(3):
            for c in range(3):
                pp = [p0.copy(), p1.copy(), p2.copy()]
                pm = [p0.copy(), p1.copy(), p2.copy()]
                pp[j][c] += h
                pm[j][c] -= h
                up, vp, _, _ = oracle.refmode_bary_uv(p, *pp)
                um, vm, _, _ = oracle.refmode_bary_uv(p, *pm)
                assert abs((up - um) / (2 * h) - du[j, c]) < 1e-6 * max(1.0, abs(du[j, c]))
                assert abs((vp - vm) / (2 * h) - dv[j, c]) < 1e-6 * max(1.0, abs(dv[j, c]))


@pytest.mark.parametrize("n,res,ert", [(8, 128, False), (16, 256, True)])
def test_reference_image_close_to_exact(oracle, n, res, ert):
    """Same fragment sets: the images differ only through the FP32 NDC depth
    (~5e-5 of view depth at distance 3), the unsigned weights outside a face
    and the a < 1e-6 drop."""
    sc = Scene(n, res, seed=n + 3, ert=ert)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)
    img_e, _, term_e, _ = oracle.render(fa, sc.pos, sc.col, cam, prm)
    img_r, term_r = oracle.refmode(fa, sc.pos, sc.col, cam, prm)
    e = np.abs(img_r - img_e)
    assert e.max() < 2e-3 and e.mean() < 2e-5, (e.max(), e.mean())
    assert (term_r == term_e).mean() > 0.999


def test_reference_adjoint_over_all_subsegments_gives_the_exact_colour_gradient(oracle):
    """Run over all four sub-segments (the reference stops at s > 0,
    Backward.glsl:222), the restated inversion and accumulateLinearConstAdjoint
    give the exact colour gradient up to the forward differences above; with
    the reference's loop bound a quarter of every segment is missing."""
    sc = Scene(8, 128, seed=11)
    fa = oracle.Faces(sc.cells, sc.pos.shape[0])
    cam, prm = sc.oracle_camera(oracle), sc.oracle_params(oracle)
    w = np.random.default_rng(5).normal(size=(128, 128, 4))
    _, gc_e = oracle.adjoint(fa, sc.pos, sc.col, cam, prm, w)
    _, _, _, gc_all = oracle.refmode(fa, sc.pos, sc.col, cam, prm, w, skip0=False)
    _, _, _, gc_ref = oracle.refmode(fa, sc.pos, sc.col, cam, prm, w)
    assert rel_err(gc_all, gc_e) < 1e-3
    assert rel_err(gc_ref, gc_e) > 0.1
