"""Generates the committed golden fixtures of this directory from the FP64 CPU
oracle (test infrastructure) and the library's .bintet writer.

    python tests/golden/make_golden.py

Fixtures
  oracle_8_128.npz    Kuhn 8^3 (seed 8, jitter 0.2), sphere camera 8, 128x128,
                      attenuation 1: FP64 image, transmittance, termination
                      index, the sorted fragment lists, and the FP64 adjoint
                      for a seeded image adjoint (normal, seed 128).
  oracle_16_512.npz   Kuhn 16^3 (seed 16), sphere camera 16, 512x512: FP64
                      image on 4096 seeded pixels, full-image sums, the list
                      offsets and a SHA-256 of the sorted records, and the
                      FP64 adjoint for a seeded image adjoint (normal, seed 512).
  single_tet_v1.bintet   the reference's SINGLE_TETRAHEDRON test case (vertex colours).
  kuhn2_cells_v2.bintet  Kuhn 2^3 with per-cell colours (version 2).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402  (test infrastructure)

from difftetvr_b200 import synthetic as S  # noqa: E402


def scene(n, res):
    cells, pos = S.kuhn_mesh(n, seed=n, jitter=0.2)
    col = S.gaussian_colors(pos, seed=n)
    view = S.sphere_camera(n)
    return cells, pos, col, view


def records_sha256(records: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(records, np.uint64).tobytes()).hexdigest()


def make_8_128():
    n, res = 8, 128
    cells, pos, col, view = scene(n, res)
    fa = O.Faces(cells, pos.shape[0])
    cam = O.make_camera(view, S.FOVY_45, res, res)
    prm = O.make_params(attenuation=1.0)
    img, tf, term, nf = O.render(fa, pos, col, cam, prm)
    off, rec = O.fragments(fa, pos, cam)
    w = np.random.default_rng(128).normal(size=(res, res, 4))
    gp, gc = O.adjoint(fa, pos, col, cam, prm, w)
    np.savez_compressed(os.path.join(HERE, "oracle_8_128.npz"), cells=cells, positions=pos, colors=col,
                        view=np.asarray(view, np.float32), res=res, image=img, transmittance=tf, termination=term,
                        offsets=off, records=rec, image_adjoint_seed=128, grad_positions=gp, grad_colors=gc)


def make_16_512():
    n, res = 16, 512
    cells, pos, col, view = scene(n, res)
    fa = O.Faces(cells, pos.shape[0])
    cam = O.make_camera(view, S.FOVY_45, res, res)
    prm = O.make_params(attenuation=1.0)
    img, tf, term, nf = O.render(fa, pos, col, cam, prm)
    off, rec = O.fragments(fa, pos, cam)
    rng = np.random.default_rng(7)
    pix = rng.choice(res * res, size=4096, replace=False)
    w = np.random.default_rng(512).normal(size=(res, res, 4))
    gp, gc = O.adjoint(fa, pos, col, cam, prm, w)
    np.savez_compressed(os.path.join(HERE, "oracle_16_512.npz"), view=np.asarray(view, np.float32), res=res,
                        pixels=pix, image_at_pixels=img.reshape(-1, 4)[pix], image_sum=img.sum(axis=(0, 1)),
                        transmittance_sum=tf.sum(), num_fragments=nf, offsets=off.astype(np.int64),
                        records_sha256=records_sha256(rec), image_adjoint_seed=512, grad_positions=gp,
                        grad_colors=gc)


def make_bintet():
    from difftetvr_b200.mesh_io import write_bintet
    # SINGLE_TETRAHEDRON (TetMesh.cpp:1017-1065)
    cells = np.array([[0, 1, 2, 3]], np.uint32)
    pos = np.array([[-0.1, -0.1, 0.1], [0.1, -0.1, 0.1], [0.0, 0.3, 0.0], [0.1, -0.1, -0.1]], np.float32)
    col = np.array([[1, 1, 1, 0.1], [1, 1, 1, 0.1], [0, 1, 0, 0.1], [1, 1, 1, 0.8]], np.float32)
    write_bintet(os.path.join(HERE, "single_tet_v1.bintet"), cells, pos, col)
    cells, pos = S.kuhn_mesh(2, seed=0, jitter=0.0)
    ccol = np.random.default_rng(2).uniform(0, 1, size=(cells.shape[0], 4)).astype(np.float32)
    write_bintet(os.path.join(HERE, "kuhn2_cells_v2.bintet"), cells, pos, None, ccol)


if __name__ == "__main__":
    make_8_128()
    make_16_512()
    make_bintet()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
