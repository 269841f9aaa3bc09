"""The autotuners' coordinate search on CPU: stand-in renderers whose timings
are a function of the configuration.  Every candidate is measured once, even
when a candidate earlier in a knob's value order than the knob's starting
value turns out fastest, and the fastest configuration is left set."""
import torch

from difftetvr_b200 import autotune


class _Tuned:
    def __init__(self, tuning):
        self.tuning = dict(tuning)

    def set_tuning(self, **cfg):
        self.tuning.update(cfg)

    def get_tuning(self):
        return dict(self.tuning)


class _Mesh:
    def __init__(self):
        self.pos = torch.zeros(4, 3, requires_grad=True)
        self.col = torch.zeros(4, 4, requires_grad=True)

    def get_vertex_positions(self):
        return self.pos

    def get_vertex_colors(self):
        return self.col

    def get_cell_colors(self):
        return None

    def get_num_cells(self):
        return 1

    def get_num_faces(self):
        return 4

    def get_color_storage(self):
        return 0


class _Renderer(_Tuned):
    def __init__(self, tuning):
        super().__init__(tuning)
        self.mesh = _Mesh()

    def get_tet_mesh(self):
        return self.mesh

    def get_viewport_size(self):
        return 8, 8

    def get_renderer_type(self):
        return 0

    def render(self):
        pass

    def render_adjoint_into(self, adj, gp, gc):
        pass


def _cost(t):
    """Synthetic time: tile 0 is fastest, then bucket sorting of every class."""
    ms = 10.0 + t["composite_tile"] + t["adjoint_tile"] if "composite_tile" in t else 10.0
    for c in autotune.SORT_CLASSES:
        ms += {"bucket": 0.0, "surrogate": 0.5, "network": 1.0}[autotune.sort_method(t, c)]
    return ms


def _patched(monkeypatch, target):
    monkeypatch.setattr(autotune, "_time_ms", lambda fn, trials: _cost(target.get_tuning()))


def _keys(timings):
    return [tuple(sorted((k, v) for k, v in t.items() if k != "ms")) for t in timings]


def test_batch_search_measures_each_candidate_once(monkeypatch):
    # Start every class on the 64-bit network (last in the value order) so
    # that "bucket", tried first, becomes the best before "network" comes up.
    br = _Tuned(dict(sort_surrogate_classes=0, sort_bucket_classes=0))
    _patched(monkeypatch, br)
    out = autotune.autotune_batch(br, views=[], trials=1, force=True)
    keys = _keys(out["timings"])
    assert len(keys) == 1 + 4 * 2 + 1 and len(set(keys)) == len(keys)
    assert out["tuning"] == dict(sort_surrogate_classes=0, sort_bucket_classes=0b111110)
    assert br.get_tuning() == out["tuning"]


def test_renderer_search_measures_each_candidate_once(monkeypatch):
    r = _Renderer(dict(composite_tile=2, adjoint_tile=2, sort_surrogate_classes=0b11110, sort_bucket_classes=0))
    _patched(monkeypatch, r)
    out = autotune.autotune_renderer(r, trials=1, force=True)
    keys = _keys(out["timings"])
    assert len(keys) == 1 + 2 + 2 + 4 * 2 + 1 and len(set(keys)) == len(keys)
    assert out["tuning"] == dict(composite_tile=0, adjoint_tile=0, sort_surrogate_classes=0,
                                 sort_bucket_classes=0b111110)
    assert r.get_tuning() == out["tuning"]
