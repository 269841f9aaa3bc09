"""Box pixel index -> (row, column) map of the warp-cooperative count pass:
row = trunc(rn(rn(k + 1/2) * rn(1/bw))) in FP32 equals floor(k / bw).  The
kernel uses it for boxes under 64 px a side (k < 2^12); it holds for every box
of at most 2^21 pixels, checked here.  FP32 arithmetic here is IEEE
round-to-nearest, as the kernel's __fadd_rn, __fmul_rn and __frcp_rn."""
import numpy as np

MAX_AREA = 1 << 21


def rows_fp32(k, bw):
    inv = np.float32(1.0) / np.float32(bw)
    return (np.float32(k).astype(np.float32) + np.float32(0.5)).astype(np.float32) * inv


def check(bw):
    bh = MAX_AREA // bw
    q = np.arange(bh, dtype=np.int64)
    # Largest rounding error sits next to the row boundaries: first and last
    # pixel of each row.
    for k in (q * bw, q * bw + bw - 1):
        kf = k.astype(np.float32)
        assert np.array_equal(kf.astype(np.int64), k)
        r = np.trunc(rows_fp32(kf, bw)).astype(np.int64)
        assert np.array_equal(r, k // bw), bw


def test_every_width_up_to_4096():
    for bw in range(1, 4097):
        check(bw)


def test_sampled_wide_boxes():
    rng = np.random.default_rng(0)
    for bw in np.unique(np.concatenate([rng.integers(4097, MAX_AREA + 1, 300), [MAX_AREA, MAX_AREA - 1, 16384]])):
        check(int(bw))


def test_all_pixels_small_widths():
    for bw in range(1, 65):
        k = np.arange(MAX_AREA - MAX_AREA % bw, dtype=np.int64)
        r = np.trunc(rows_fp32(k.astype(np.float32), bw)).astype(np.int64)
        assert np.array_equal(r, k // bw), bw


# ---------------------------------------------------------------------------
# Exact row spans (row_span / span_edge): per box row, the FP32 estimate of
# each edge's column bound corrected by one exact integer test on each side
# must give exactly the pixels whose centres pass the three edge tests.

def _edges(ax, ay):
    """EdgeT set() for the counter-clockwise edges 1->2, 2->0, 0->1 (int64)."""
    out = []
    for a, b in ((1, 2), (2, 0), (0, 1)):
        dx, dy = ax[:, b] - ax[:, a], ay[:, b] - ay[:, a]
        t = ((dy < 0) | ((dy == 0) & (dx > 0))).astype(np.int64)
        base = dy * ax[:, a] - dx * ay[:, a] + t - 1
        out.append((base, -dy * 256, dx * 256))
    return out


def _span_edge(base, sx, sy, r, bw, lo, hi):
    q = base + sy * r
    zero = sx == 0
    lo = np.where(zero & (q < 0), bw, lo)
    hi = np.where(zero & (q < 0), -1, hi)
    inv = np.where(zero, np.float32(0), np.float32(1) / np.where(zero, 1, sx).astype(np.float32))
    b = (-(q.astype(np.float32)) * inv).astype(np.float32)
    b = np.minimum(np.maximum(b, np.float32(-2)), (bw + 1).astype(np.float32))
    T = lambda c: q + sx * c
    up = np.ceil(b).astype(np.int64)
    up = np.where(T(up - 1) >= 0, up - 1, np.where(T(up) < 0, up + 1, up))
    dn = np.floor(b).astype(np.int64)
    dn = np.where(T(dn + 1) >= 0, dn + 1, np.where(T(dn) < 0, dn - 1, dn))
    lo = np.where(~zero & (sx > 0), np.maximum(lo, up), lo)
    hi = np.where(~zero & (sx < 0), np.minimum(hi, dn), hi)
    return lo, hi


def _check_spans(rng, n, extent):
    # Vertices in 1/256 px relative to the centre of the box's first pixel.
    ax = rng.integers(-128, extent, size=(n, 3)).astype(np.int64)
    ay = rng.integers(-128, extent, size=(n, 3)).astype(np.int64)
    area = (ax[:, 1] - ax[:, 0]) * (ay[:, 2] - ay[:, 0]) - (ay[:, 1] - ay[:, 0]) * (ax[:, 2] - ax[:, 0])
    keep = area > 0  # counter-clockwise as set up by raster_setup (front faces are swapped)
    ax, ay = ax[keep], ay[keep]
    bw = np.full(len(ax), extent // 256 + 2, np.int64)
    edges = _edges(ax, ay)
    for r in range(int(bw[0])):
        lo, hi = np.zeros(len(ax), np.int64), bw - 1
        for base, sx, sy in edges:
            lo, hi = _span_edge(base, sx, sy, r, bw, lo, hi)
        for c in range(int(bw[0])):
            inside = np.ones(len(ax), bool)
            for base, sx, sy in edges:
                inside &= base + sx * c + sy * r >= 0
            assert np.array_equal(inside, (lo <= c) & (c <= hi)), (r, c)


def test_row_spans_are_exact_small_boxes():
    _check_spans(np.random.default_rng(1), 20000, 63 * 256)


def test_row_spans_are_exact_thin_and_wide_boxes():
    rng = np.random.default_rng(2)
    _check_spans(rng, 4000, 300 * 256)
    # Slivers: nearly collinear vertices, where the bounds are ill-conditioned.
    n = 20000
    ax = rng.integers(0, 40 * 256, size=(n, 1)) + np.array([[0, 5000, 10000]]) + rng.integers(-3, 4, size=(n, 3))
    ay = rng.integers(0, 40 * 256, size=(n, 1)) + np.array([[0, 3, 7]]) + rng.integers(-3, 4, size=(n, 3))
    ax, ay = ax.astype(np.int64), ay.astype(np.int64)
    area = (ax[:, 1] - ax[:, 0]) * (ay[:, 2] - ay[:, 0]) - (ay[:, 1] - ay[:, 0]) * (ax[:, 2] - ax[:, 0])
    sw = area < 0
    ax[sw, 1], ax[sw, 2] = ax[sw, 2].copy(), ax[sw, 1].copy()
    ay[sw, 1], ay[sw, 2] = ay[sw, 2].copy(), ay[sw, 1].copy()
    edges = _edges(ax, ay)
    bw = np.full(n, 90, np.int64)
    for r in range(90):
        lo, hi = np.zeros(n, np.int64), bw - 1
        for base, sx, sy in edges:
            lo, hi = _span_edge(base, sx, sy, r, bw, lo, hi)
        for c in range(90):
            inside = np.ones(n, bool)
            for base, sx, sy in edges:
                inside &= base + sx * c + sy * r >= 0
            assert np.array_equal(inside, (lo <= c) & (c <= hi)), (r, c)
