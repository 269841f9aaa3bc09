"""difftetvr_b200 — B200-native (sm_100a) differentiable tetrahedral volume
rendering with the API of the `difftetvr` module of chrismile/DiffTetVR.

    import difftetvr_b200 as d
    mesh = d.TetMesh(); mesh.set_use_gradients(True)
    mesh.set_hex_mesh_const(d.AABB3(d.vec3(-1,-1,-1), d.vec3(1,1,1)), 17, 17, 17, d.vec4(.5,.5,.5,.1))
    r = d.Renderer(d.RendererType.PPLL); r.set_tet_mesh(mesh); r.set_viewport_size(512, 512)
    image = d.DifferentiableRenderer(r)()      # [H, W, 4] premultiplied RGBA on CUDA
"""
from .types import (AABB3, ColorStorage, RendererType, SplitGradientType, TestCase, uvec3, vec3,  # noqa: F401
                    vec4)
from .tet_mesh import TetMesh, build_faces_host, build_hex_mesh, convert_hex_to_tet_indices  # noqa: F401
from .renderer import Renderer  # noqa: F401
from .pyutils import DifferentiableRenderer, DifferentiableRenderingFunction  # noqa: F401
from .regularizer import TetRegularizer  # noqa: F401

__version__ = "0.1.0"


def set_device_type(device_type: str) -> None:
    """set_device_type (Module.cpp:1171-1173).  Only CUDA devices are supported."""
    if str(device_type) != "cuda":
        raise RuntimeError("difftetvr_b200 runs on CUDA devices only (no CPU fallback)")
