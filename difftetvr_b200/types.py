"""Small value types and enums of the `difftetvr` module
(src/Module/Module.cpp:706-771, src/Module/difftetvr.pyi)."""
from __future__ import annotations

import enum


class vec3:  # noqa: N801 - reference name
    def __init__(self, x: float, y: float, z: float):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __repr__(self):
        return f"vec3({self.x}, {self.y}, {self.z})"


class vec4:  # noqa: N801
    def __init__(self, x: float, y: float, z: float, w: float):
        self.x, self.y, self.z, self.w = float(x), float(y), float(z), float(w)

    def __iter__(self):
        return iter((self.x, self.y, self.z, self.w))

    def __repr__(self):
        return f"vec4({self.x}, {self.y}, {self.z}, {self.w})"


class uvec3:  # noqa: N801
    def __init__(self, x: int, y: int, z: int):
        self.x, self.y, self.z = int(x), int(y), int(z)

    def __iter__(self):
        return iter((self.x, self.y, self.z))


class AABB3:
    """Axis-aligned box (sgl::AABB3 as bound in Module.cpp:727-737)."""

    def __init__(self, min: vec3 | None = None, max: vec3 | None = None):  # noqa: A002
        self.min = min if min is not None else vec3(0.0, 0.0, 0.0)
        self.max = max if max is not None else vec3(0.0, 0.0, 0.0)

    def get_dimensions(self) -> vec3:
        return vec3(self.max.x - self.min.x, self.max.y - self.min.y, self.max.z - self.min.z)

    def get_extent(self) -> vec3:
        d = self.get_dimensions()
        return vec3(0.5 * d.x, 0.5 * d.y, 0.5 * d.z)

    def get_center(self) -> vec3:
        return vec3(0.5 * (self.min.x + self.max.x), 0.5 * (self.min.y + self.max.y),
                    0.5 * (self.min.z + self.max.z))

    def get_minimum(self) -> vec3:
        return self.min

    def get_maximum(self) -> vec3:
        return self.max


class TestCase(enum.IntEnum):
    __test__ = False  # not a pytest class
    SINGLE_TETRAHEDRON = 0
    CUBE_CENTRAL_GRADIENT = 1


class ColorStorage(enum.IntEnum):
    PER_VERTEX = 0
    PER_CELL = 1


class RendererType(enum.IntEnum):
    PPLL = 0
    PROJECTION = 1
    INTERSECTION = 2


class SplitGradientType(enum.IntEnum):
    POSITION = 0
    COLOR = 1
    ABS_POSITION = 2
    ABS_COLOR = 3
