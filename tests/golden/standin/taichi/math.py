"""ti.math for the serial stand-in: vector types and the few helpers the
reference uses.  TEST INFRASTRUCTURE ONLY (see the package docstring)."""
from __future__ import annotations

import taichi as _ti

vec2 = _ti.VectorType(2, _ti.f32)
vec3 = _ti.VectorType(3, _ti.f32)
vec4 = _ti.VectorType(4, _ti.f32)
ivec2 = _ti.VectorType(2, _ti.i32)
ivec3 = _ti.VectorType(3, _ti.i32)
ivec4 = _ti.VectorType(4, _ti.i32)


def clamp(x, lo, hi):
    return _ti.min(_ti.max(x, lo), hi)


def dot(a, b):
    return a.dot(b)


def length(a):
    return a.norm()


def normalize(a):
    return a.normalized()
