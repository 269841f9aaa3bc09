"""Host-side parts of the reference-facing API that need no GPU: the
reference's linked-list export layout built from offsets + sorted records,
and set_device_type."""
import numpy as np
import pytest

import difftetvr_b200 as d
from difftetvr_b200.renderer import linked_list_view


def _walk(nodes, head):
    out, i = [], int(head)
    while i != -1:
        out.append(i)
        nxt = int(np.int32(nodes[i, 2].view(np.int32)))
        i = nxt
    return out


def test_linked_list_view_walks_every_list_in_order():
    rng = np.random.default_rng(3)
    w, h = 5, 4
    counts = rng.integers(0, 4, size=w * h)
    counts[[0, 7, 19]] = 0  # empty pixels, first and last included
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    n = int(offsets[-1])
    depth = np.sort(rng.uniform(1.0, 3.0, size=n)).astype(np.float32)
    lo = rng.integers(0, 1 << 30, size=n, dtype=np.uint64)
    records = (depth.view(np.uint32).astype(np.uint64) << np.uint64(32)) | lo
    nodes, heads = linked_list_view(offsets, records, w, h)
    assert nodes.shape == (n, 3) and nodes.dtype == np.uint32 and heads.shape == (h, w)
    for p in range(w * h):
        head = heads.reshape(-1)[p]
        if counts[p] == 0:
            assert head == -1
            continue
        idx = _walk(nodes, head)
        assert idx == list(range(int(offsets[p]), int(offsets[p + 1])))
        np.testing.assert_array_equal(nodes[idx, 0], (records[idx] & np.uint64(0xFFFFFFFF)).astype(np.uint32))
        np.testing.assert_array_equal(nodes[idx, 1].view(np.float32), depth[idx])


def test_set_device_type():
    d.set_device_type("cuda")
    with pytest.raises(RuntimeError):
        d.set_device_type("cpu")
