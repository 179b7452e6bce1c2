"""Uneven solves built from batch specs (scenes.batch_spec) and run as one batch graph (gi_batch_*) or one by one.

A Solve owns a resident scene, voxel world and cascades for one seeded spec: the scene on the device, the frame set,
the G-buffer drawn on the device, the voxel windows placed at the camera.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

from . import configs, frame as fr, gpu, scenes


@dataclass
class Solve:
    spec: dict
    scene: scenes.Scene
    sg: gpu.SceneGpu
    vox: gpu.VoxWorld
    rc: gpu.Rc
    frame: object

    def destroy(self):
        for h in (self.rc, self.vox, self.sg):
            h.destroy()


def solve_params(spec: dict, atlas: str = "f32"):
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": spec["cascades"]})
    G, L = spec["G"], spec["levels"]
    v = configs.vox_params({"v0": spec["v0"], "levels": L, "G": G, "maxBricks": min(L * G ** 3, 32768),
                            "maxVoxels": 1 << 21})
    return p, v


def make_solve(ctx: gpu.Context, spec: dict, atlas: str = "f32", stream=None, scene: scenes.Scene = None) -> Solve:
    s = scene or scenes.mixed_scene(spec["seed"], spec["tris"])
    p, v = solve_params(spec, atlas)
    W, H = spec["width"], spec["height"]
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=s.sun_e, sky=s.sky,
                                     cascades=p.cascades, P=p.P))
    sg = gpu.SceneGpu(ctx, s)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    rc.set_frame(F, stream)
    rc.render_gbuffer(sg, stream)
    vw.update(s.camera.eye)
    return Solve(spec, s, sg, vw, rc, F)


def make_batch(ctx: gpu.Context, solves: List[Solve], stream) -> gpu.Batch:
    b = gpu.Batch(ctx, [x.rc for x in solves], [x.vox for x in solves])
    b.capture(stream)
    return b
