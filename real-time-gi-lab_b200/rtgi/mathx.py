"""Host-side camera and matrix math with the reference's exact arithmetic (src/core/math.ts, src/core/frame.ts).

The reference computes in JavaScript numbers (IEEE f64) and stores into Float32Array (round to nearest even).  The
functions here evaluate the same expressions in the same order in Python floats (f64) and round to f32 where the
reference stores into a Float32Array, so a frame packed here is bit-identical to the reference's packFrame for the
same camera.  ``hypot`` follows V8's Math.hypot (Kahan-compensated sum of squares scaled by the largest value).
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np

Vec3 = Sequence[float]


def f32(x: float) -> float:
    """Round a double to the nearest f32 (what a Float32Array store does)."""
    return float(np.float32(x))


def hypot(*xs: float) -> float:
    """Math.hypot as V8 evaluates it (max scaling, Kahan-compensated sum)."""
    if not xs:
        return 0.0
    absv = []
    mx = 0.0
    nan = False
    for v in xs:
        if v != v:
            nan = True
            absv.append(0.0)
            continue
        a = abs(v)
        absv.append(a)
        if a > mx:
            mx = a
    if mx == math.inf:
        return math.inf
    if nan:
        return math.nan
    if mx == 0:
        return 0.0
    s = 0.0
    comp = 0.0
    for a in absv:
        n = a / mx
        summand = n * n - comp
        prelim = s + summand
        comp = (prelim - s) - summand
        s = prelim
    return math.sqrt(s) * mx


def sub(a: Vec3, b: Vec3) -> list[float]:
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def add3(a: Vec3, b: Vec3) -> list[float]:
    return [a[0] + b[0], a[1] + b[1], a[2] + b[2]]


def scale3(a: Vec3, s: float) -> list[float]:
    return [a[0] * s, a[1] * s, a[2] * s]


def cross(a: Vec3, b: Vec3) -> list[float]:
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def dot(a: Vec3, b: Vec3) -> float:
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def normalize(a: Vec3) -> list[float]:
    l = hypot(a[0], a[1], a[2])
    return [a[0] / l, a[1] / l, a[2] / l]


def mat_mul(a: Sequence[float], b: Sequence[float]) -> list[float]:
    """mul (math.ts:13-22): column-major a * b, f64 sums of the f32 inputs, stored as f32."""
    r = [0.0] * 16
    for c in range(4):
        for row in range(4):
            s = 0.0
            for k in range(4):
                s += a[k * 4 + row] * b[c * 4 + k]
            r[c * 4 + row] = f32(s)
    return r


def look_at(eye: Vec3, target: Vec3, up: Vec3) -> list[float]:
    """lookAt (math.ts:24-34)."""
    f = normalize(sub(target, eye))
    s = normalize(cross(f, up))
    u = cross(s, f)
    vals = [s[0], u[0], -f[0], 0, s[1], u[1], -f[1], 0, s[2], u[2], -f[2], 0, -dot(s, eye), -dot(u, eye), dot(f, eye), 1]
    return [f32(v) for v in vals]


def ortho_zo(half_w: float, half_h: float, near: float, far: float) -> list[float]:
    """orthoZO (math.ts:102-109): depth 0 at near, 1 at far."""
    return [f32(v) for v in [1 / half_w, 0, 0, 0, 0, 1 / half_h, 0, 0, 0, 0, -1 / (far - near), 0, 0, 0,
                             -near / (far - near), 1]]


def perspective_reversed_infinite(fov_y: float, aspect: float, near: float) -> list[float]:
    """perspectiveReversedInfinite (math.ts:37-45): depth 1 at the near plane, 0 at infinity."""
    f = 1 / math.tan(fov_y / 2)
    return [f32(v) for v in [f / aspect, 0, 0, 0, 0, f, 0, 0, 0, 0, 0, -1, 0, 0, near, 0]]


def invert(m: Sequence[float]) -> list[float]:
    """General 4x4 inverse (math.ts:79-99): cofactors in f64 of the f32 inputs, each divided by the determinant."""
    inv = [0.0] * 16
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10]
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10]
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9]
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9]
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10]
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10]
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9]
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9]
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6]
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6]
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5]
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5]
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6]
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6]
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5]
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5]
    det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12]
    return [f32(v / det) for v in inv]
