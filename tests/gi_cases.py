"""Parity cases shared by the tests: the two benchmark configurations plus lit and overflow variants that make every
branch of the path carry non-zero values (config 0's two cascades stop short of its lamp, so its irradiance is 0)."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from rtgi import configs, frame as fr, scenes


@dataclass
class Case:
    name: str
    scene: scenes.Scene
    width: int
    height: int
    vox: configs.VoxParams
    rc: configs.RcParams
    frame: np.ndarray = field(default=None)
    shadow: int = 0          # sun shadow map size (0: none, every voxel's sun visibility 1)


def _frame(scene, W, H, p: configs.RcParams, sun_e=None, sky=None, shadow=False):
    lvp, bias = [0.0] * 16, (0.0, 0.0)
    if shadow:   # the sun's view-projection over the scene bounds (lighting.ts:100-106), one layer
        bmin, bmax = fr.scene_bounds(scene.positions)
        lvp, bias = fr.scene_sun_view_proj(bmin, bmax, scene.sun_dir), fr.SHADOW_BIAS
    return fr.pack_frame(fr.FrameParams(cam=scene.camera, width=W, height=H, sun_dir=scene.sun_dir,
                                        sun_e=scene.sun_e if sun_e is None else sun_e,
                                        sky=scene.sky if sky is None else sky, cascades=p.cascades, P=p.P,
                                        s_min=p.sMin, lift=p.lift, light_view_proj=lvp, shadow_bias=bias))


def config0(atlas: str = "f32") -> Case:
    """Room of 200 boxes, 1 level of 64^3 voxels of 0.16 m, 256x256, 2 cascades, DDA cap 64."""
    s = scenes.room_scene(0)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda64", {"cascades": 2})
    v = configs.vox_params({"v0": 0.16, "levels": 1, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 18})
    c = Case("config0", s, 256, 256, v, p)
    c.frame = _frame(s, 256, 256, p)
    return c


def config1(atlas: str = "f32", width: int = 1920, height: int = 1080) -> Case:
    """Colonnade of ~260k triangles, 4 levels of 128^3 voxels from 0.1 m, 1920x1080, 5 cascades, DDA cap 256, the
    sun's 4096^2 shadow map (voxSun)."""
    s = scenes.colonnade_scene(0)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": 5})
    v = configs.vox_params({"v0": 0.1, "levels": 4, "G": 16, "maxBricks": 16384, "maxVoxels": 1 << 22})
    c = Case("config1", s, width, height, v, p, shadow=fr.SHADOW_SIZE)
    c.frame = _frame(s, width, height, p, shadow=True)
    return c


def room_lit(atlas: str = "f16") -> Case:
    """The room under sun and sky, 3 levels (reduce, voxLevelFor), 5 cascades (merge of every kind)."""
    s = scenes.room_scene(0)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": 5})
    v = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    c = Case("room_lit", s, 320, 240, v, p)
    c.frame = _frame(s, 320, 240, p, sun_e=fr.SUN_E, sky=fr.SKY)
    return c


def leak(t: float = 0.1, atlas: str = "bf16") -> Case:
    """The reference's leak room (scenes.ts:261) with its recorded voxel parameters, 5 cascades, sun and sky."""
    s = scenes.leak_room(t)
    p = configs.parse_config(f"screen-8-voxel-{atlas}", {"cascades": 5})
    v = configs.vox_params({"v0": 0.1, "levels": 5, "G": 64, "maxBricks": 32768, "maxVoxels": 4194304})
    c = Case(f"leak-{t}", s, 320, 180, v, p)
    c.frame = _frame(s, 320, 180, p, sun_e=fr.SUN_E, sky=fr.SKY)
    return c


def leak_sun(t: float = 0.1, atlas: str = "f32", size: int = 1024) -> Case:
    """The leak room with the sun's shadow map (voxSun): sunlight through the openings only."""
    c = leak(t, atlas)
    c.name, c.shadow = f"leak-sun-{t}", size
    c.frame = _frame(c.scene, c.width, c.height, c.rc, sun_e=fr.SUN_E, sky=fr.SKY, shadow=True)
    return c


def empty(atlas: str = "f32") -> Case:
    """No triangles: an empty clipmap, a background-only G-buffer (no valid probe), at a ragged 100 x 37."""
    s = scenes.Scene("empty", np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 4), np.uint32),
                     [scenes.Material("grey", (0.5, 0.5, 0.5, 1.0))], scenes.Camera((0, 1.7, 5), (0, 1, 0), 60, 0.05),
                     sun_dir=(0.3, 1.0, 0.2), sun_e=fr.SUN_E, sky=fr.SKY)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda64", {"cascades": 3})
    v = configs.vox_params({"v0": 0.16, "levels": 2, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 16})
    c = Case("empty", s, 100, 37, v, p)
    c.frame = _frame(s, 100, 37, p)
    return c


def single_triangle(atlas: str = "f32") -> Case:
    """One large triangle filling part of the view under sun and sky (the rest background), at a ragged 123 x 61."""
    b = scenes.Builder([scenes.Material("grey", (0.7, 0.6, 0.5, 1.0))])
    b.quad([-3, 0, 3], [3, 0, 3], [3, 0, -3], [-3, 0, -3])
    s0 = b.scene("tri", scenes.Camera((0, 1.7, 5), (0, 0, 0), 60, 0.05), sun_dir=(0.3, 1.0, 0.2), sun_e=fr.SUN_E,
                 sky=fr.SKY)
    s = scenes.Scene("single-triangle", s0.positions, s0.normals, s0.tri[:1].copy(), s0.materials, s0.camera,
                     sun_dir=s0.sun_dir, sun_e=s0.sun_e, sky=s0.sky)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda64", {"cascades": 3})
    v = configs.vox_params({"v0": 0.08, "levels": 2, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 16})
    c = Case("single-triangle", s, 123, 61, v, p, shadow=256)
    c.frame = _frame(s, 123, 61, p, shadow=True)
    return c


def tiny(atlas: str = "f16") -> Case:
    """room_lit at 7 x 5 pixels: a single probe per cascade, smaller than the 8-pixel probe cell."""
    c = room_lit(atlas)
    c.name, c.width, c.height = "tiny", 7, 5
    c.frame = _frame(c.scene, 7, 5, c.rc, sun_e=fr.SUN_E, sky=fr.SKY)
    return c


def overflow(atlas: str = "f32") -> Case:
    """room_lit with pools too small: dropped bricks (read at the coarser level) and voxels without attributes."""
    c = room_lit(atlas)
    c.name = "overflow"
    c.vox = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 300, "maxVoxels": 20000})
    return c
