"""Committed golden fixtures (tests/golden/, made by make_golden.py): the oracle
still reproduces them, and the .bintet reader/writer follows the file layout
of the reference's BinTetLoader / BinTetWriter byte for byte."""
import hashlib
import os
import struct

import numpy as np
import pytest

from difftetvr_b200 import synthetic as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_oracle_reproduces_8_128(oracle):
    g = load("oracle_8_128.npz")
    res = int(g["res"])
    fa = oracle.Faces(g["cells"], g["positions"].shape[0])
    cam = oracle.make_camera(g["view"].tolist(), S.FOVY_45, res, res)
    prm = oracle.make_params(attenuation=1.0)
    img, tf, term, nf = oracle.render(fa, g["positions"], g["colors"], cam, prm)
    np.testing.assert_array_equal(img, g["image"])
    np.testing.assert_array_equal(term, g["termination"])
    off, rec = oracle.fragments(fa, g["positions"], cam)
    np.testing.assert_array_equal(off, g["offsets"])
    np.testing.assert_array_equal(rec, g["records"])
    w = np.random.default_rng(int(g["image_adjoint_seed"])).normal(size=(res, res, 4))
    gp, gc = oracle.adjoint(fa, g["positions"], g["colors"], cam, prm, w)
    # Per-thread partial sums: equal up to FP64 summation order.
    np.testing.assert_allclose(gp, g["grad_positions"], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(gc, g["grad_colors"], rtol=1e-10, atol=1e-14)


def test_oracle_reproduces_16_512_lists_and_samples(oracle):
    g = load("oracle_16_512.npz")
    res = int(g["res"])
    cells, pos = S.kuhn_mesh(16, seed=16, jitter=0.2)
    col = S.gaussian_colors(pos, seed=16)
    fa = oracle.Faces(cells, pos.shape[0])
    cam = oracle.make_camera(g["view"].tolist(), S.FOVY_45, res, res)
    off, rec = oracle.fragments(fa, pos, cam)
    np.testing.assert_array_equal(off, g["offsets"])
    assert hashlib.sha256(rec.tobytes()).hexdigest() == str(g["records_sha256"])
    img = oracle.render(fa, pos, col, cam, oracle.make_params(attenuation=1.0))[0]
    np.testing.assert_array_equal(img.reshape(-1, 4)[g["pixels"]], g["image_at_pixels"])


# -- .bintet ------------------------------------------------------------------
def _pack_bintet(version, cells, pos, vcol, ccol=None):
    b = struct.pack("<I", version)
    for arr, per in ((cells.reshape(-1).astype("<u4"), 1), (pos.astype("<f4"), 3), (vcol.astype("<f4"), 4)):
        b += struct.pack("<I", arr.size // per) + arr.tobytes()
    if version == 2:
        b += struct.pack("<I", ccol.shape[0]) + ccol.astype("<f4").tobytes()
    return b


def test_bintet_fixture_layout_single_tet():
    from difftetvr_b200.mesh_io import peek_bintet, read_bintet
    path = os.path.join(GOLDEN, "single_tet_v1.bintet")
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    pos = np.array([[-0.1, -0.1, 0.1], [0.1, -0.1, 0.1], [0.0, 0.3, 0.0], [0.1, -0.1, -0.1]], np.float32)
    col = np.array([[1, 1, 1, 0.1], [1, 1, 1, 0.1], [0, 1, 0, 0.1], [1, 1, 1, 0.8]], np.float32)
    with open(path, "rb") as f:
        assert f.read() == _pack_bintet(1, cells, pos, col)
    h = peek_bintet(path)
    assert h == {"version": 1, "num_cells": 1, "num_vertices": 4, "num_vertex_colors": 4, "num_cell_colors": 0}
    c2, p2, v2, cc2, ver = read_bintet(path)
    assert ver == 1 and cc2 is None
    np.testing.assert_array_equal(c2, cells)
    np.testing.assert_array_equal(p2, pos)
    np.testing.assert_array_equal(v2, col)


def test_bintet_fixture_cell_colours_v2():
    from difftetvr_b200.mesh_io import read_bintet
    cells, pos = S.kuhn_mesh(2, seed=0, jitter=0.0)
    ccol = np.random.default_rng(2).uniform(0, 1, size=(cells.shape[0], 4)).astype(np.float32)
    path = os.path.join(GOLDEN, "kuhn2_cells_v2.bintet")
    with open(path, "rb") as f:
        assert f.read() == _pack_bintet(2, cells, pos, np.zeros((0, 4), np.float32), ccol)
    c2, p2, v2, cc2, ver = read_bintet(path)
    assert ver == 2 and v2.shape == (0, 4)
    np.testing.assert_array_equal(c2, cells)
    np.testing.assert_array_equal(p2, pos)
    np.testing.assert_array_equal(cc2, ccol)


def test_bintet_round_trip_and_errors(tmp_path):
    from difftetvr_b200._lib import DTV_ERR_ARG, DtvError
    from difftetvr_b200.mesh_io import read_bintet, write_bintet
    cells, pos = S.kuhn_mesh(3, seed=4)
    col = S.gaussian_colors(pos, seed=4)
    p = str(tmp_path / "m.bintet")
    write_bintet(p, cells, pos, col)
    c2, p2, v2, cc2, ver = read_bintet(p)
    assert ver == 1
    np.testing.assert_array_equal(c2, cells)
    np.testing.assert_array_equal(p2, pos)
    np.testing.assert_array_equal(v2, col)
    data = open(p, "rb").read()
    for bad, what in ((data[:-5], "truncated"), (struct.pack("<I", 3) + data[4:], "version"),
                      (data[:4] + struct.pack("<I", 7) + data[8:], "cell count")):
        q = str(tmp_path / "bad.bintet")
        open(q, "wb").write(bad)
        with pytest.raises(DtvError) as e:
            read_bintet(q)
        assert e.value.code == DTV_ERR_ARG, what
    with pytest.raises(DtvError):
        read_bintet(str(tmp_path / "missing.bintet"))


def test_linked_list_view_of_the_fixture_lists():
    """The reference-layout view (PPLL nodes + heads) of the 8^3 fixture lists:
    following next from each head visits exactly the pixel's sorted records."""
    from difftetvr_b200.renderer import linked_list_view
    g = load("oracle_8_128.npz")
    off, rec = g["offsets"], g["records"]
    nodes, heads = linked_list_view(off, rec, 128, 128)
    assert nodes.shape == (rec.shape[0], 3) and heads.shape == (128, 128)
    flat = heads.reshape(-1)
    for p in np.flatnonzero(np.diff(off) > 0)[::97]:
        i, walked = int(flat[p]), []
        while i != -1:
            walked.append((int(nodes[i, 1]) << 32) | int(nodes[i, 0]))
            nx = int(nodes[i, 2])
            i = -1 if nx == 0xFFFFFFFF else nx
        assert walked == [int(x) for x in rec[off[p]:off[p + 1]]]
    assert np.all(flat[np.diff(off) == 0] == -1)
    depth = nodes[:, 1].view(np.float32)
    assert np.all(depth > 0)
