"""Autotuner: picks the kernel configuration of a renderer (pixel tile of the
composite and adjoint blocks, sort method per list-length class) or of a batch
renderer (sort method per class) by timing the candidates on the caller's own
workload with CUDA events.  Every configuration gives identical results, so
the search only changes speed.  Coordinate search: each knob in turn, the
others held at their best value so far.  Results are cached per workload key
(resolution, mesh size, renderer type, colour storage)."""
from __future__ import annotations

import torch

TILES = (0, 1, 2)               # composite 16x16, 32x8, 8x32 (256 threads); adjoint 16x8, 32x4, 8x16 (128)
SORT_CLASSES = (1, 2, 3, 4, 5)  # lists of up to 64, 128, 256, 512, 1024 records
SORT_METHODS = ("bucket", "surrogate", "network")


def methods_for(c: int) -> tuple:
    """Sort methods available to list-length class c (no surrogate keys for
    the shared-memory class 5)."""
    return SORT_METHODS if c <= 4 else ("bucket", "network")


def sort_method(tuning: dict, c: int) -> str:
    """Sort method of list-length class c under `tuning` (bucket bits win)."""
    if (tuning["sort_bucket_classes"] >> c) & 1:
        return "bucket"
    return "surrogate" if (tuning["sort_surrogate_classes"] >> c) & 1 else "network"


def with_sort_method(tuning: dict, c: int, method: str) -> dict:
    """`tuning` with class c switched to `method`."""
    bit = 1 << c
    b = tuning["sort_bucket_classes"] & ~bit
    q = tuning["sort_surrogate_classes"] & ~bit
    if method == "bucket":
        b |= bit
    elif method == "surrogate":
        q |= bit
    return dict(tuning, sort_bucket_classes=b, sort_surrogate_classes=q)

_cache: dict = {}


def _time_ms(fn, trials: int) -> float:
    fn()  # warm-up (first-use allocations)
    best = float("inf")
    for _ in range(trials):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _key(renderer) -> tuple:
    mesh = renderer.get_tet_mesh()
    w, h = renderer.get_viewport_size()
    return ("renderer", int(renderer.get_renderer_type()), w, h, mesh.get_num_cells(), mesh.get_num_faces(),
            int(mesh.get_color_storage()))


def autotune_renderer(renderer, trials: int = 3, force: bool = False) -> dict:
    """Times render (+ adjoint when the mesh uses gradients) for each candidate
    and leaves the fastest configuration set on the renderer.  Returns
    {"tuning": ..., "ms": ..., "timings": [...]}."""
    key = _key(renderer)
    if not force and key in _cache:
        renderer.set_tuning(**_cache[key]["tuning"])
        return _cache[key]
    mesh = renderer.get_tet_mesh()
    pos = mesh.get_vertex_positions()
    w, h = renderer.get_viewport_size()
    adj = torch.full((h, w, 4), 1e-3, device=pos.device)
    cells = mesh.get_cell_colors() if mesh.get_cell_colors() is not None else mesh.get_vertex_colors()
    gp = torch.zeros_like(pos.detach())
    gc = torch.zeros_like(cells.detach())
    with_adjoint = pos.requires_grad

    def step():
        renderer.render()
        if with_adjoint:
            renderer.render_adjoint_into(adj, gp, gc)

    timings = []

    def measure(**cfg):
        renderer.set_tuning(**cfg)
        ms = _time_ms(step, trials)
        timings.append({**renderer.get_tuning(), "ms": ms})
        return ms

    best = renderer.get_tuning()
    best_ms = measure(**best)
    # Each knob's starting value was measured with the configuration before
    # it, so it is skipped even when another value has become the best.
    for knob, values in (("composite_tile", TILES), ("adjoint_tile", TILES if with_adjoint else (best["adjoint_tile"],))):
        start = best[knob]
        for v in values:
            if v == start:
                continue
            cand = dict(best, **{knob: v})
            ms = measure(**cand)
            if ms < best_ms:
                best, best_ms = cand, ms
    for c in SORT_CLASSES:
        start = sort_method(best, c)
        for method in methods_for(c):
            if method == start:
                continue
            cand = with_sort_method(best, c, method)
            ms = measure(**cand)
            if ms < best_ms:
                best, best_ms = cand, ms
    renderer.set_tuning(**best)
    out = {"tuning": best, "ms": best_ms, "timings": timings}
    _cache[key] = out
    return out


def autotune_batch(batch_renderer, views, trials: int = 2, force: bool = False) -> dict:
    """Times BatchRenderer.render(views) for each sort method per list-length
    class (depth buckets, surrogate keys, 64-bit network) and leaves the
    fastest set.  Returns {"tuning": ..., "ms": ...}."""
    key = ("batch", tuple((v.mesh, v.width, v.height) for v in views))
    if not force and key in _cache:
        batch_renderer.set_tuning(**_cache[key]["tuning"])
        return _cache[key]
    timings = []

    def measure(cfg):
        batch_renderer.set_tuning(**cfg)
        ms = _time_ms(lambda: batch_renderer.render(views), trials)
        timings.append({**cfg, "ms": ms})
        return ms

    best = batch_renderer.get_tuning()
    best_ms = measure(best)
    for c in SORT_CLASSES:
        start = sort_method(best, c)  # measured already (see autotune_renderer)
        for method in methods_for(c):
            if method == start:
                continue
            cand = with_sort_method(best, c, method)
            ms = measure(cand)
            if ms < best_ms:
                best, best_ms = cand, ms
    batch_renderer.set_tuning(**best)
    out = {"tuning": best, "ms": best_ms, "timings": timings}
    _cache[key] = out
    return out
