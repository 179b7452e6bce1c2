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
    movers: tuple = None     # (rtgi.movers.MovingObjects, t): objects posed on the device before the G-buffer


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


def batch_shape(name: str, seed: int, tris: int, G: int, levels: int, v0: float, W: int, H: int, cascades: int,
                atlas: str) -> Case:
    """A solve of the batching / serving distribution (rtgi.batch.solve_params): the procedural box/column mix, its
    clipmap shape, resolution and cascade count."""
    s = scenes.mixed_scene(seed, tris)
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": cascades})
    v = configs.vox_params({"v0": v0, "levels": levels, "G": G, "maxBricks": min(levels * G ** 3, 32768),
                            "maxVoxels": 1 << 21})
    c = Case(name, s, W, H, v, p)
    c.frame = _frame(s, W, H, p)
    return c


def batch_g4_l1() -> Case:
    return batch_shape("batch-g4-l1", 7, 20_000, 4, 1, 0.2, 320, 180, 2, "f32")


def batch_g4_l4() -> Case:
    return batch_shape("batch-g4-l4", 8, 30_000, 4, 4, 0.15, 320, 180, 4, "f16")


def batch_g32_l1() -> Case:
    return batch_shape("batch-g32-l1", 9, 40_000, 32, 1, 0.1, 480, 270, 3, "f32")


def batch_g32_l4() -> Case:
    """4 levels of 256^3 voxels (131,072 brick pointers per rebuild), f16 atlas, 5 cascades."""
    return batch_shape("batch-g32-l4", 10, 60_000, 32, 4, 0.1, 480, 270, 5, "f16")


def posed(scene: scenes.Scene, objs, t: float) -> scenes.Scene:
    """The scene with its moving objects posed at t as gi_scene_rigid_apply poses them on the device: each vertex
    through its object's 3x4 transform, ((m0 x + m1 y) + m2 z) + m3 in f32 per row."""
    import dataclasses
    m = objs.transforms(t)
    per, n = objs.per, objs.centres.shape[0]
    P = scene.positions.astype(np.float32).copy()
    N = scene.normals.astype(np.float32).copy()
    rest_p = P[objs.first:objs.first + per * n].reshape(n, per, 3)
    rest_n = N[objs.first:objs.first + per * n].reshape(n, per, 3)
    M = m.reshape(n, 1, 12)
    out_p = np.empty_like(rest_p)
    out_n = np.empty_like(rest_n)
    for r in range(3):
        out_p[..., r] = ((M[..., 4 * r] * rest_p[..., 0] + M[..., 4 * r + 1] * rest_p[..., 1])
                         + M[..., 4 * r + 2] * rest_p[..., 2]) + M[..., 4 * r + 3]
        out_n[..., r] = (M[..., 4 * r] * rest_n[..., 0] + M[..., 4 * r + 1] * rest_n[..., 1]) + M[..., 4 * r + 2] * rest_n[..., 2]
    P[objs.first:objs.first + per * n] = out_p.reshape(-1, 3)
    N[objs.first:objs.first + per * n] = out_n.reshape(-1, 3)
    return dataclasses.replace(scene, positions=P, normals=N)


def movers_f16() -> Case:
    """A serving request: the box/column mix with 80 moving boxes posed on the device (gi_scene_rigid_apply) at
    t = 0.6 s, f16 atlas, 2 levels of 128^3, 320 x 180, 3 cascades.  The oracle gets the same poses from `posed`."""
    from rtgi import movers
    base = scenes.mixed_scene(5, 25_000)
    s, objs = movers.with_moving_boxes(base, 80, scenes.PCG32(17, stream=3))
    c = batch_shape("movers-f16", 5, 25_000, 16, 2, 0.1, 320, 180, 3, "f16")
    c.scene, c.movers = s, (objs, 0.6)
    c.frame = _frame(s, c.width, c.height, c.rc)
    return c


def toon(style: bool = True, atlas: str = "f32") -> Case:
    """room_lit with every other box material toon (flag 4): their hits inject style.ts's emission-side operator
    (toonSun, rc.ts:114) while the frame's style word is on, Lambert when it is off."""
    import dataclasses
    c = room_lit(atlas)
    mats = [dataclasses.replace(m, flags=m.flags | scenes.FLAG_TOON) if m.name.startswith("box") and i % 2 else m
            for i, m in enumerate(c.scene.materials)]
    c.scene = dataclasses.replace(c.scene, materials=mats)
    c.name = "toon" if style else "toon-style-off"
    c.frame = _frame(c.scene, c.width, c.height, c.rc, sun_e=fr.SUN_E, sky=fr.SKY)
    if not style:
        c.frame[136] = 0.0
    return c
