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
