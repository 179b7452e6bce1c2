"""The per-frame uniform (src/core/frame.ts): Camera, cameraMatrices, packFrame, octSolidAngles.

``pack_frame`` returns the 640-byte Frame block the GI path reads (frame.ts:4-21), word for word as the reference's
packFrame (frame.ts:76-94) lays it out; the C-ABI takes it unchanged (gi_rc_set_frame).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import mathx

FRAME_BYTES = 160 * 4
SUN_E = (9.0, 8.5, 7.8)          # rcrun.ts:26
SKY = (0.45, 0.6, 0.9)           # rcrun.ts:27

# Word offsets of the Frame fields (frame.ts:5-20).
F_VIEWPROJ, F_INVVIEWPROJ, F_EYE, F_FWD, F_SUNDIR, F_SUNE, F_SKY, F_SIZE = 0, 16, 80, 84, 88, 92, 96, 100
F_RC, F_RC2, F_RU, F_RU2, F_OMEGA, F_STYLE = 104, 108, 112, 116, 120, 136


SHADOW_SIZE = 4096               # createLighting's shadowSize (lighting.ts:113)
SHADOW_BIAS = (0.0002, 0.0)      # one layer: the comparison bias of layer 0 (lighting.ts:134)


def scene_sun_view_proj(bounds_min, bounds_max, sun_dir) -> list:
    """sceneSunViewProj (lighting.ts:100-106): the sun's orthographic view-projection over the scene's bounding
    sphere, depth 0 on the sunward side of the sphere and 1 on the far side."""
    center = mathx.scale3(mathx.add3(bounds_min, bounds_max), 0.5)
    radius = mathx.hypot(*mathx.sub(bounds_max, bounds_min)) / 2
    d = mathx.scale3(sun_dir, 1 / mathx.hypot(*sun_dir))
    up = [0, 0, 1] if abs(d[1]) > 0.99 else [0, 1, 0]
    return mathx.mat_mul(mathx.ortho_zo(radius, radius, 0, 2 * radius),
                         mathx.look_at(mathx.add3(center, mathx.scale3(d, radius)), center, up))


# The camera-following shadow layers of an instanced world (lighting.ts:93-96): layer 0 of half width NEAR_R m, layer 1
# of FAR_R m, depth DEPTH_R m on either side of the camera along the sun; biases in metres over the 2 DEPTH_R range
SHADOW_NEAR_R, SHADOW_FAR_R, SHADOW_DEPTH_R = 32, 410, 300
SHADOW_WORLD_BIAS = (0.012 / (2 * SHADOW_DEPTH_R), 0.15 / (2 * SHADOW_DEPTH_R))


def _js_round(x: float) -> float:
    """Math.round: the nearest integer, halves toward +infinity (exact, unlike floor(x + 0.5) near 0.5)."""
    r = math.floor(x)
    return float(r + 1 if x - r >= 0.5 else r)


def world_sun_view_projs(sun_dir, eye, size: int = SHADOW_SIZE) -> tuple:
    """cameraMatrix (lighting.ts:115-123) for layer 0 (NEAR_R) and layer 1 (FAR_R): an orthographic light view of
    half width r centred on the camera, the centre snapped to the layer's texels across the sun (so the map does not
    shimmer as the camera moves), depth 0 DEPTH_R m sunward of the camera and 1 DEPTH_R m past it."""
    sun = mathx.scale3(sun_dir, 1 / mathx.hypot(*sun_dir))
    up0 = [0, 0, 1] if abs(sun[1]) > 0.99 else [0, 1, 0]
    right = mathx.normalize(mathx.cross(up0, sun))
    up = mathx.cross(sun, right)

    def layer(r):
        texel = 2 * r / size
        snap = lambda x: _js_round(x / texel) * texel
        c = mathx.add3(mathx.add3(mathx.scale3(right, snap(mathx.dot(eye, right))), mathx.scale3(up, snap(mathx.dot(eye, up)))),
                       mathx.scale3(sun, mathx.dot(eye, sun)))
        return mathx.mat_mul(mathx.ortho_zo(r, r, 0, 2 * SHADOW_DEPTH_R),
                             mathx.look_at(mathx.add3(c, mathx.scale3(sun, SHADOW_DEPTH_R)), c, up0))
    return layer(SHADOW_NEAR_R), layer(SHADOW_FAR_R)


def scene_bounds(positions) -> tuple:
    """boundsMin / boundsMax (gltf.ts:147) of f32 vertex positions, as f64 values."""
    p = np.asarray(positions, dtype=np.float32)
    return [float(x) for x in p.min(axis=0)], [float(x) for x in p.max(axis=0)]


@dataclass
class Camera:
    eye: tuple
    target: tuple
    fov_y_deg: float
    near: float


def camera_matrices(c: Camera, width: int, height: int) -> dict:
    """cameraMatrices (frame.ts:58-63)."""
    view = mathx.look_at(c.eye, c.target, [0, 1, 0])
    proj = mathx.perspective_reversed_infinite(c.fov_y_deg * math.pi / 180, width / height, c.near)
    view_proj = mathx.mat_mul(proj, view)
    return {"view": view, "viewProj": view_proj, "invViewProj": mathx.invert(view_proj),
            "fwd": mathx.normalize(mathx.sub(c.target, c.eye))}


_OMEGA_CACHE: dict = {}


def oct_solid_angles(res: int = 4, samples: int = 1 << 20) -> np.ndarray:
    """octSolidAngles (frame.ts:105-114): per octahedral texel, the share of 2^20 Fibonacci-sphere points x 4 pi."""
    key = (res, samples)
    if key in _OMEGA_CACHE:
        return _OMEGA_CACHE[key].copy()
    golden = math.pi * (3 - math.sqrt(5))
    i = np.arange(samples, dtype=np.float64)
    z = 1 - (2 * i + 1) / samples
    r = np.sqrt(1 - z * z)
    phi = golden * i
    x, y = r * np.cos(phi), r * np.sin(phi)
    s = np.abs(x) + np.abs(y) + np.abs(z)
    u, v = x / s, y / s
    neg = z < 0
    ou, ov = u.copy(), v.copy()
    u = np.where(neg, (1 - np.abs(ov)) * np.where(ou >= 0, 1.0, -1.0), u)
    v = np.where(neg, (1 - np.abs(ou)) * np.where(ov >= 0, 1.0, -1.0), v)
    u, v = u * 0.5 + 0.5, v * 0.5 + 0.5
    tx = np.minimum(res - 1, np.floor(u * res)).astype(np.int64)
    ty = np.minimum(res - 1, np.floor(v * res)).astype(np.int64)
    counts = np.bincount(ty * res + tx, minlength=res * res).astype(np.float64)
    out = (counts / samples * 4 * math.pi).astype(np.float32)
    _OMEGA_CACHE[key] = out
    return out.copy()


@dataclass
class FrameParams:
    """FrameParams (frame.ts:65-74)."""
    cam: Camera
    width: int
    height: int
    prev_cam: Optional[Camera] = None
    light_view_proj: Sequence[float] = field(default_factory=lambda: [0.0] * 16)
    shadow_far: Optional[Sequence[float]] = None
    shadow_bias: tuple = (0.0, 0.0)
    sun_dir: tuple = (0.0, 1.0, 0.0)
    sun_e: tuple = (0.0, 0.0, 0.0)
    sky: tuple = (0.0, 0.0, 0.0)
    s_min: float = 0.05
    P: float = 8
    lift: float = 0.25
    thickness_min: float = 0.15
    px_stride: float = 4
    exposure: float = 1.0
    cascades: int = 5
    slot: int = 0
    reg_stride: int = 1
    max_steps: int = 16
    ray_stride: int = 1
    seed: int = 0
    prev_valid: bool = False
    analytic: bool = False
    omega0: Optional[np.ndarray] = None
    style: tuple = (1.0, 1.0, 0.0)


def pack_frame(p: FrameParams) -> np.ndarray:
    """packFrame (frame.ts:76-94) -> 160 words (float32 view; the u32 fields are bit patterns)."""
    buf = np.zeros(160, dtype=np.float32)
    u = buf.view(np.uint32)
    cur = camera_matrices(p.cam, p.width, p.height)
    prev = camera_matrices(p.prev_cam or p.cam, p.width, p.height)
    buf[0:16] = cur["viewProj"]
    buf[16:32] = cur["invViewProj"]
    buf[32:48] = prev["viewProj"]
    buf[48:64] = prev["invViewProj"]
    buf[64:80] = np.asarray(p.light_view_proj, dtype=np.float64)
    buf[80:84] = [*p.cam.eye, p.cam.near]
    buf[84:88] = [*cur["fwd"], 0]
    buf[88:92] = [*mathx.normalize(p.sun_dir), 0]
    buf[92:96] = [*p.sun_e, 0]
    buf[96:100] = [*p.sky, 0]
    buf[100:104] = [p.width, p.height, 1 / p.width, 1 / p.height]
    pix_ang = 2 * math.tan(p.cam.fov_y_deg * math.pi / 360) / p.height
    buf[104:108] = [p.s_min, pix_ang, p.P, 0]
    buf[108:112] = [p.lift, p.thickness_min, p.px_stride, p.exposure]
    u[112:116] = [p.cascades, p.slot, p.reg_stride, p.max_steps]
    u[116:120] = [p.ray_stride, p.seed, 1 if p.prev_valid else 0, 1 if p.analytic else 0]
    omega = p.omega0 if p.omega0 is not None else oct_solid_angles(4)
    buf[120:136] = omega
    buf[136:140] = [*p.style, 0]
    if p.shadow_far is not None:
        buf[140:156] = np.asarray(p.shadow_far, dtype=np.float64)
    buf[156:160] = [2 if p.shadow_far is not None else 1, p.shadow_bias[0], p.shadow_bias[1], 0]
    return buf
