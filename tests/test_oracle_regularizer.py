"""Pinning the oracle's tet-quality regularizer on the CPU: known values of the
quality measure, FP64 central differences of the penalty, the reference's
denominator clamp, and the mirrored softplus direction (inverted tets are
pushed back)."""
import numpy as np
import pytest

from difftetvr_b200 import synthetic as S

REGULAR = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], np.float64)


def _quality(p):
    """6 sqrt(2) V / l_rms^3 with the reference's sign of V."""
    D = np.linalg.det(np.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]]))
    S_ = sum(np.sum((p[a] - p[b]) ** 2) for a in range(4) for b in range(a + 1, 4))
    return 6 * np.sqrt(2) * (-D / 6) / (S_ / 6) ** 1.5


def test_quality_of_regular_tet_is_one_in_reference_orientation(oracle):
    """The regular tetrahedron scores |q| = 1; the orientation with negative
    det (the Kuhn cells' orientation) has q = +1 and a small penalty, the
    mirrored one q = -1 and a large one."""
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    p = REGULAR if np.linalg.det(np.stack([REGULAR[i] - REGULAR[0] for i in (1, 2, 3)])) < 0 else REGULAR[[0, 2, 1, 3]]
    assert abs(_quality(p) - 1.0) < 1e-12
    lam, beta = 2.0, 3.0
    good, _ = oracle.tet_regularizer(cells, p, lam, beta)
    bad, _ = oracle.tet_regularizer(cells, p[[0, 2, 1, 3]], lam, beta)
    np.testing.assert_allclose(good, lam / beta * np.log1p(np.exp(-beta)), rtol=1e-12)
    np.testing.assert_allclose(bad, lam / beta * np.log1p(np.exp(beta)), rtol=1e-12)


def test_kuhn_cells_have_positive_quality(oracle):
    cells, pos = S.kuhn_mesh(3, seed=1)
    q = np.array([_quality(pos[c].astype(np.float64)) for c in cells])
    assert np.all(q > 0.1)


@pytest.mark.parametrize("scale", [1.0, 0.2])
def test_gradient_matches_central_differences(oracle, scale):
    """Unclamped tets (S^(5/2) > 1e-5): the analytic gradient equals FP64
    central differences of the summed penalty, including inverted tets."""
    cells, pos = S.kuhn_mesh(3, seed=2, jitter=0.45)
    pos = pos.astype(np.float64) * scale
    rng = np.random.default_rng(0)
    pos[21] += rng.normal(size=3) * 0.6 * scale  # invert some cells around an interior vertex
    lam, beta = 0.7, 4.0
    _, grad = oracle.tet_regularizer(cells, pos, lam, beta)
    h = 1e-6 * scale
    for v, k in [(21, 0), (21, 2), (5, 1), (40, 0), (13, 2), (30, 1)]:
        xp, xm = pos.copy(), pos.copy()
        xp[v, k] += h
        xm[v, k] -= h
        fd = (oracle.tet_regularizer(cells, xp, lam, beta)[0] - oracle.tet_regularizer(cells, xm, lam, beta)[0]) / (2 * h)
        assert abs(fd - grad[v, k]) <= 1e-6 * max(1.0, abs(fd)), (v, k, fd, grad[v, k])


def test_denominator_clamp_scales_small_tets(oracle):
    """For S^(5/2) < 1e-5 the reference divides by 1e-5 instead: the gradient of
    a tiny tet is the true one times S^(5/2) / 1e-5."""
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    p = REGULAR[[0, 2, 1, 3]] * 0.01 + 0.3
    S_ = sum(np.sum((p[a] - p[b]) ** 2) for a in range(4) for b in range(a + 1, 4))
    assert S_ ** 2.5 < 1e-5
    p = p.copy()
    p[3] += [0.002, -0.001, 0.0015]
    lam, beta = 1.0, 2.0
    _, g = oracle.tet_regularizer(cells, p, lam, beta)
    h = 1e-9
    xp, xm = p.copy(), p.copy()
    xp[3, 0] += h
    xm[3, 0] -= h
    fd = (oracle.tet_regularizer(cells, xp, lam, beta)[0] - oracle.tet_regularizer(cells, xm, lam, beta)[0]) / (2 * h)
    S_ = sum(np.sum((p[a] - p[b]) ** 2) for a in range(4) for b in range(a + 1, 4))
    np.testing.assert_allclose(g[3, 0], fd * S_ ** 2.5 / 1e-5, rtol=1e-5)


def test_descent_restores_inverted_tet(oracle):
    """A slightly inverted, nearly flat tet (apex pushed just through the
    opposite face) is pushed back to positive quality by gradient descent."""
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    base = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.3, 1.0, 0.0]])
    p = np.vstack([base, [0.4, 0.3, 0.05]])
    if _quality(p) > 0:
        p[3, 2] = -0.05
    assert -0.3 < _quality(p) < 0
    for _ in range(400):
        _, g = oracle.tet_regularizer(cells, p, 1.0, 2.0)
        p -= 0.05 * g
    assert _quality(p) > 0
