"""The radiance-cascade runner's entry (src/native/rc.ts with src/core/rcrun.ts runConfig and src/runner/report.ts) for
the path this library runs: `--scene` and `--configs` as the reference takes them, per config a timed static run of
the GI passes (voxel rebuild, giBuild, giTrace, giMerge, giGather) and a `<config>.summary.json` beside the logged
lines.  What the reference's runner does besides (moving-camera metrics, images, DDGI and WebGL2 comparators, the
triangle-BVH tracer) is not part of this path.

    python -m rtgi.rcrun --scene colonnade --configs screen-8-voxel-f16,screen-8-voxel-f32-dda256 --frames 240

Scenes: the seeded procedural scenes of this library (`room`, `colonnade`, `leak-<t>` as scenes.ts leakRoom,
`mix-<seed>` of the batch distribution, each optionally `-obj<N>` with N moving boxes posed at --pose-frame).
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import sys
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import configs, frame as fr, scenes

PASSES = ("vox", "giBuild", "giTrace", "giMerge", "giGather")


def stats(ms: Sequence[float]) -> dict:
    """stats (rcrun.ts:114-118): median, mean, p05, p95, p99, max, rounded to 1e-3 ms."""
    s = sorted(ms)
    def pct(q):
        if not s:
            return 0.0
        i = q * (len(s) - 1)
        lo, hi = int(math.floor(i)), int(math.ceil(i))
        return s[lo] + (s[hi] - s[lo]) * (i - lo)
    r = lambda x: round(x * 1000) / 1000
    return {"median": r(pct(0.5)), "mean": r(sum(s) / max(1, len(s))), "p05": r(pct(0.05)), "p95": r(pct(0.95)),
            "p99": r(pct(0.99)), "max": r(s[-1] if s else 0.0)}


def load_scene(name: str, pose_frame: float = 0.0, fps: float = 30.0):
    """A scene by name; `-obj<N>` adds N moving boxes posed at frame pose_frame.  Returns (scene, voxel defaults)."""
    base, _, objs = name.partition("-obj")
    if base == "room":
        s, vox = scenes.room_scene(0), {"v0": 0.16, "levels": 1, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 18}
    elif base == "colonnade":
        s, vox = scenes.colonnade_scene(0), {"v0": 0.1, "levels": 4, "G": 16, "maxBricks": 16384, "maxVoxels": 1 << 22}
    elif base.startswith("leak-"):
        s, vox = scenes.leak_room(float(base[5:])), {"v0": 0.1, "levels": 5, "G": 64, "maxBricks": 32768,
                                                     "maxVoxels": 1 << 22}
    elif base.startswith("mix-"):
        spec = scenes.batch_spec(int(base[4:]))
        s = scenes.mixed_scene(spec["seed"], spec["tris"])
        vox = {"v0": spec["v0"], "levels": spec["levels"], "G": spec["G"],
               "maxBricks": min(spec["levels"] * spec["G"] ** 3, 32768), "maxVoxels": 1 << 21}
    else:
        raise ValueError(f"unknown scene {name}")
    if objs:
        from .movers import with_moving_boxes
        s, movers = with_moving_boxes(s, int(objs), scenes.PCG32(7, stream=41))
        pos, nrm = movers.pose(pose_frame / fps)
        s.positions = s.positions.copy()
        s.normals = s.normals.copy()
        s.positions[movers.first:] = pos
        s.normals[movers.first:] = nrm
    return s, vox


def run_config(ctx, sg, scene, name: str, p: configs.RcParams, vp: configs.VoxParams, width: int, height: int,
               warmup: int, frames: int, sky, log=print, shadow_size: int = fr.SHADOW_SIZE) -> dict:
    """runConfig (rcrun.ts) for one config, static camera: warm-up frames, then `frames` timed solves (per-pass CUDA
    events), the DDA statistics of one more solve, the probe and voxel counters.  As the reference's renderer: the
    sun's shadow map over the scene (shadow_size 0: none) and multi-bounce when the config has it on (the default)."""
    from . import gpu
    lvp, bias = [0.0] * 16, (0.0, 0.0)
    if shadow_size:
        bmin, bmax = fr.scene_bounds(scene.positions)
        lvp, bias = fr.scene_sun_view_proj(bmin, bmax, scene.sun_dir), fr.SHADOW_BIAS
    F = fr.pack_frame(fr.FrameParams(cam=scene.camera, width=width, height=height, sun_dir=scene.sun_dir,
                                     sun_e=scene.sun_e, sky=sky, cascades=p.cascades, P=p.P, s_min=p.sMin, lift=p.lift,
                                     light_view_proj=lvp, shadow_bias=bias))
    vw = gpu.VoxWorld(sg, vp)
    rc = gpu.Rc(ctx, p, width, height)
    try:
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        if shadow_size:
            rc.render_shadow(sg, shadow_size)
        if p.bounce:
            rc.set_bounce(vw)
        vw.update(scene.camera.eye)
        for _ in range(warmup):
            rc.solve(vw)
        rc.set_timing(True)
        per = {k: [] for k in PASSES}
        for _ in range(frames):
            rc.solve(vw)
            for k, v in rc.pass_times().items():
                per[k].append(v)
        rc.set_timing(False)
        timing = {k: stats(v) for k, v in per.items()}
        timing["giTotal"] = stats([sum(x) for x in zip(*[per[k] for k in PASSES])])
        rc.set_stats(1)
        rc.solve(vw)
        c = rc.read_counts()
        rc.set_stats(0)
        tracer = [{"intervals": int(c[24 + i]), "meanSteps": round(float(c[32 + i]) / c[24 + i], 4) if c[24 + i] else 0,
                   "atStepCap": int(c[64 + i])} for i in range(p.cascades)]
        vc = vw.read_counters()
        vox = {k: vc[k] for k in ("bricks", "voxels", "brickOverflow", "bigOverflow", "voxelOverflow", "bricksPerLevel",
                                  "bigPerLevel")}
        irr = rc.read_irradiance()
        out = {"config": name, "params": dataclasses.asdict(p), "voxParams": dataclasses.asdict(vp),
               "shadowMap": shadow_size, "bounce": bool(p.bounce),
               "resolution": f"{width}x{height}", "allocatedBytes": rc.bytes(), "voxAllocatedBytes": vw.bytes(),
               "static": {"timing": timing, "counts": [int(x) for x in c[:p.cascades]], "vox": vox},
               "tracer": tracer, "_irr": irr}
        t = timing
        log(f"  GI static {t['giTotal']['median']} ms (vox {t['vox']['median']}, build {t['giBuild']['median']}, "
            f"trace {t['giTrace']['median']}, merge {t['giMerge']['median']}, gather {t['giGather']['median']})")
        log(f"  probes {', '.join(str(x) for x in out['static']['counts'])}; allocated "
            f"{rc.bytes() / 2 ** 20:.1f} MiB, vox {vw.bytes() / 2 ** 20:.1f} MiB")
        log(f"  vox {json.dumps(vox)}")
        log(f"  tracer {json.dumps(tracer)}")
        return out
    finally:
        rc.destroy()
        vw.destroy()


def pack_irradiance(irr: np.ndarray) -> np.ndarray:
    """packIrradiance (runner/report.ts:54-58): rgb + tag per pixel as float32, rows top to bottom; the tag is 1 for a
    valid pixel and 0 for the background (this path has no toon tag)."""
    f = np.array(irr, np.float32).reshape(-1, 4).copy()
    f[:, 3] = (f[:, 3] > 0).astype(np.float32)
    return f


def vox_bench(ctx, sg, scene, vp: configs.VoxParams, frames: int = 60) -> dict:
    """--vox-bench: the voxel rebuild alone, timed with CUDA events around each rebuild."""
    import torch
    from . import gpu
    vw = gpu.VoxWorld(sg, vp)
    st = torch.cuda.current_stream()
    try:
        vw.update(scene.camera.eye)
        for _ in range(5):
            vw.encode(st)
        ms = []
        for _ in range(frames):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            vw.encode(st)
            e1.record(st)
            st.synchronize()
            ms.append(e0.elapsed_time(e1))
        vc = vw.read_counters()
        return {"frames": frames, "total": stats(ms), "bricks": vc["bricks"], "voxels": vc["voxels"],
                "bricksPerLevel": vc["bricksPerLevel"], "bigPerLevel": vc["bigPerLevel"]}
    finally:
        vw.destroy()


def main(argv: Optional[List[str]] = None) -> int:
    ap = argparse.ArgumentParser(prog="rtgi.rcrun", description=__doc__.splitlines()[0])
    ap.add_argument("--scene", default="colonnade")
    ap.add_argument("--configs", default="screen-8-voxel")
    ap.add_argument("--frames", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=60)
    ap.add_argument("--out", default=None)
    ap.add_argument("--no-sky", action="store_true")
    ap.add_argument("--params", default="{}", help="RcParams overrides (JSON)")
    ap.add_argument("--vox", default="{}", help="VoxParams overrides (JSON; unknown keys are an error)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--pose-frame", type=float, default=0.0)
    ap.add_argument("--dump-irr", action="store_true")
    ap.add_argument("--vox-bench", action="store_true")
    ap.add_argument("--tag", default="default")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--shadow-size", type=int, default=fr.SHADOW_SIZE, help="sun shadow map size (0: no sun visibility)")
    ap.add_argument("--no-bounce", action="store_true", help="multi-bounce off whatever the config says")
    a = ap.parse_args(argv)
    overrides = json.loads(a.params)
    parsed = [(c, configs.parse_config(c, overrides)) for c in a.configs.split(",")]
    if a.no_bounce:
        parsed = [(c, dataclasses.replace(p, bounce=False)) for c, p in parsed]
    t0 = time.perf_counter()
    scene, vox_defaults = load_scene(a.scene, a.pose_frame)
    vp = configs.vox_params({**vox_defaults, **json.loads(a.vox)})
    out_dir = a.out or os.path.join("out", "rc", a.scene)
    os.makedirs(out_dir, exist_ok=True)
    from . import gpu
    ctx = gpu.Context(a.device)
    sg = gpu.SceneGpu(ctx, scene)
    lo, hi = scene.positions.min(0), scene.positions.max(0)
    print(f"scene {scene.name}: {scene.triangle_count} triangles, loaded in {round((time.perf_counter() - t0) * 1000)} ms; "
          f"bounds {','.join(f'{x:.2f}' for x in lo)} .. {','.join(f'{x:.2f}' for x in hi)}", flush=True)
    try:
        if a.vox_bench:
            r = vox_bench(ctx, sg, scene, vp)
            print(json.dumps(r), flush=True)
            with open(os.path.join(out_dir, f"vox-bench.{a.tag}.json"), "w") as f:
                json.dump({"scene": {"name": scene.name, "triangles": scene.triangle_count},
                           "voxParams": dataclasses.asdict(vp), **r}, f, indent=2)
            return 0
        sky = (0.0, 0.0, 0.0) if a.no_sky else scene.sky
        for name, p in parsed:
            print(name, flush=True)
            r = run_config(ctx, sg, scene, name, p, vp, a.width, a.height, a.warmup, a.frames, sky,
                           log=lambda s: print(s, flush=True), shadow_size=a.shadow_size)
            irr = r.pop("_irr")
            if a.dump_irr:
                pack_irradiance(irr).tofile(os.path.join(out_dir, f"{name}.static.irr.f32"))
            summary = {"scene": {"name": scene.name, "triangles": scene.triangle_count, "sunDir": list(scene.sun_dir)},
                       "frames": {"warmup": a.warmup, "measured": a.frames}, "sky": list(sky), **r}
            with open(os.path.join(out_dir, f"{name}.summary.json"), "w") as f:
                json.dump(summary, f, indent=2)
    finally:
        sg.destroy()
        ctx.destroy()
    return 0


if __name__ == "__main__":
    sys.exit(main())
