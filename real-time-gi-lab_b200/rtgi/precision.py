"""Atlas precision study: the irradiance of f32, f16 and bf16 cascade atlases against the FP64 reference of the merge
and gather (gi_rc_merge_gather_f64), over frames of a scene with moving boxes whose clipmap is rebuilt every frame.
Modes "f16"/"bf16" also store the SH and the irradiance in 16 bits (the reference's f16 storage); "-f32out" keeps
those two in f32, so only the atlas and the merge are in 16 bits.

The reference stores its atlases, SH and irradiance in f16 (rc.ts:309-310, 768-773, 1073) with f32 arithmetic; this
study states what that storage costs.  All atlas modes trace the same intervals with the same f32 arithmetic, so the
FP64 reference starts from the f32 atlas's traced intervals, which are exactly the f16/bf16 modes' values before
they are rounded for storage.  Error statistics are computed on the device with torch (plumbing only).
"""
from __future__ import annotations

import math
from typing import Dict, Sequence

import numpy as np

from . import configs, frame as fr, gpu, scenes
from .movers import with_moving_boxes

# moving boxes in the colonnade's aisles in front of the camera (centre x, centre z, half extent x, half extent z)
BOX_AREA = (13.0, -1.0, 10.0, 7.0)


def precision_scene(seed: int = 0, n_boxes: int = 64):
    """The colonnade with n_boxes rigid boxes (half sides 0.1-0.5 m, speeds U(0, 2) m/s, spin U(-1, 1) rad/s)."""
    return with_moving_boxes(scenes.colonnade_scene(seed), n_boxes, scenes.PCG32(seed, stream=41), area=BOX_AREA)


def colonnade_params(atlas: str, width: int = 1920, height: int = 1080):
    """The colonnade workload's clipmap (4 levels x 128^3 voxels from 0.1 m) and cascades (5, DDA cap 256).  atlas: a
    storage mode, optionally with "-f32out" (SH and irradiance kept in f32)."""
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": 5})
    v = configs.vox_params({"v0": 0.1, "levels": 4, "G": 16, "maxBricks": 16384, "maxVoxels": 1 << 22})
    return p, v


class ErrorStats:
    """Relative error of one atlas mode, accumulated over frames on the device.

    Per valid pixel (FP64 alpha 1) and colour channel: e = |x - x64| / max(|x64|, tau), tau = 1e-3 x the frame's mean
    |x64| (so near-black pixels are measured against the frame's scale, not divided by ~0).  Quantiles come from a
    histogram of log10(e) in 0.1-decade bins and are reported as the bin's upper edge."""
    LO, HI, BINS = -12.0, 1.0, 130

    def __init__(self, torch, device):
        self.t = torch
        self.hist = torch.zeros(self.BINS + 2, dtype=torch.int64, device=device)
        self.sq_err = self.sq_ref = self.sum_rel = self.max_rel = 0.0
        self.n = self.alpha_mismatch = self.frames = 0

    def add(self, x, ref):
        t = self.t
        x = x.to(t.float64)
        valid = ref[..., 3] > 0
        self.alpha_mismatch += int(((x[..., 3] > 0) != valid).sum().item())
        r = ref[..., :3][valid]
        y = x[..., :3][valid]
        self.frames += 1
        if r.numel() == 0:
            return
        tau = 1e-3 * float(r.abs().mean().item())
        d = (y - r).abs()
        rel = d / t.clamp(r.abs(), min=max(tau, 1e-300))
        lg = t.log10(rel.clamp_min(1e-300))
        idx = t.clamp(t.floor((lg - self.LO) / (self.HI - self.LO) * self.BINS), -1, self.BINS).to(t.int64) + 1
        self.hist += t.bincount(idx.reshape(-1), minlength=self.BINS + 2)
        self.sq_err += float((d * d).sum().item())
        self.sq_ref += float((r * r).sum().item())
        self.sum_rel += float(rel.sum().item())
        self.max_rel = max(self.max_rel, float(rel.max().item()))
        self.n += rel.numel()

    def quantile(self, q: float) -> float:
        h = self.hist.cpu().numpy()
        c = np.cumsum(h)
        if c[-1] == 0:
            return 0.0
        k = int(np.searchsorted(c, q * c[-1]))
        if k == 0:
            return 10.0 ** self.LO
        return 10.0 ** (self.LO + k * (self.HI - self.LO) / self.BINS)

    def summary(self) -> Dict[str, float]:
        return {"rel_l2": math.sqrt(self.sq_err / self.sq_ref) if self.sq_ref > 0 else 0.0,
                "mean_rel": self.sum_rel / max(1, self.n), "p50_rel": self.quantile(0.5),
                "p99_rel": self.quantile(0.99), "p999_rel": self.quantile(0.999), "max_rel": self.max_rel,
                "values": self.n, "frames": self.frames, "alpha_mismatch": self.alpha_mismatch}


# storage-rounding study: cascades whose atlas storage is rounded to f16 with every stage in double
# (gi_rc_merge_gather_f64_rounded), named by the cascades rounded
ROUNDED = {"c0": 0b00001, "c4": 0b10000, "c3-c4": 0b11000, "c2-c4": 0b11100, "c1-c4": 0b11110, "c0-c4": 0b11111}


def run(ctx: gpu.Context, frames: int = 100, dt: float = 1.0 / 30.0,
        atlases: Sequence[str] = ("f32", "f16", "bf16", "f16-f32out", "bf16-f32out"),
        seed: int = 0, n_boxes: int = 64, width: int = 1920, height: int = 1080, device: int = 0,
        shadow_size: int = fr.SHADOW_SIZE, rounded: Dict[str, int] = ROUNDED) -> dict:
    """The study: per frame, pose the boxes, draw the sun's shadow map (the boxes move; shadow_size 0: no sun
    visibility), rebuild the clipmap with voxSun, solve the cascades in every atlas mode, run the FP64 merge and
    gather from the f32 mode's trace, and accumulate each mode's irradiance error.  Also times each mode's cascade
    solve (CUDA events on the solve stream; median over frames).

    rounded: the storage-rounding study, per entry a bit mask of cascades whose atlas storage (traced intervals and,
    above cascade 0, merged radiances) is rounded to f16 while every stage stays in double; its error against the
    exact FP64 result is the storage's alone, without the f32 arithmetic, and its atlas bytes are stated beside it."""
    import torch
    dev = torch.device("cuda", device)
    stream = torch.cuda.current_stream(dev)
    s, objs = precision_scene(seed, n_boxes)
    sg = gpu.SceneGpu(ctx, s)
    rcs = {}
    vox = None
    try:
        for a in atlases:
            p, v = colonnade_params(a, width, height)
            if vox is None:
                vox = gpu.VoxWorld(sg, v)
            rcs[a] = gpu.Rc(ctx, p, width, height)
        if "f32" not in rcs:
            raise ValueError("the FP64 reference starts from the f32 atlas's trace: include 'f32'")
        rcs["f32"].set_debug_hits(True)
        lvp, bias = [0.0] * 16, (0.0, 0.0)
        if shadow_size:   # the light covers the scene's bounds at rest (the boxes stay inside the colonnade)
            bmin, bmax = fr.scene_bounds(s.positions)
            lvp, bias = fr.scene_sun_view_proj(bmin, bmax, s.sun_dir), fr.SHADOW_BIAS
        F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=width, height=height, sun_dir=s.sun_dir, sun_e=s.sun_e,
                                         sky=s.sky, cascades=rcs["f32"].params.cascades, P=rcs["f32"].params.P,
                                         light_view_proj=lvp, shadow_bias=bias))
        for rc in rcs.values():
            rc.set_frame(F, stream)
        vox.update(s.camera.eye)
        ref = torch.empty((height, width, 4), dtype=torch.float64, device=dev)
        outs = {a: torch.empty((height, width, 4), device=dev,
                               dtype=torch.float32 if rc.irr_bytes() == 16 * width * height else torch.float16)
                for a, rc in rcs.items()}
        stats = {a: ErrorStats(torch, dev) for a in rcs}
        rstats = {k: ErrorStats(torch, dev) for k in rounded}
        tmp = torch.empty((height, width, 4), dtype=torch.float64, device=dev) if rounded else None
        times = {a: [] for a in rcs}
        counters = []
        for f in range(frames):
            pos, nrm = objs.pose(f * dt)
            sg.update_vertices(objs.first, pos, nrm, stream)
            if shadow_size:
                rcs["f32"].render_shadow(sg, shadow_size, stream)
            vox.encode(stream, sun_rc=rcs["f32"] if shadow_size else None)
            ev = {}
            for a, rc in rcs.items():
                rc.render_gbuffer(sg, stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rc.encode(vox, stream)
                e1.record(stream)
                ev[a] = (e0, e1)
                rc.read_irradiance_async(outs[a].data_ptr(), stream)
            rcs["f32"].merge_gather_f64(stream)
            rcs["f32"].read_irradiance_f64(ref.data_ptr(), stream)
            for a in rcs:
                stats[a].add(outs[a], ref)
            for k, mask in rounded.items():
                rcs["f32"].merge_gather_f64(stream, f16_cascades=mask)
                rcs["f32"].read_irradiance_f64(tmp.data_ptr(), stream)
                rstats[k].add(tmp, ref)
            stream.synchronize()
            for a, (e0, e1) in ev.items():
                times[a].append(e0.elapsed_time(e1))
            if f == 0 or f == frames - 1:
                counters.append(vox.read_counters(stream))
        out = {a: dict(stats[a].summary(), solve_ms=float(np.median(times[a]))) for a in rcs}
        lay = configs.cascade_layout(rcs["f32"].params, width, height)
        rays = [c["tiles_x"] * c["tiles_y"] * c["res"] ** 2 for c in lay["casc"]]
        r_out = {k: dict(rstats[k].summary(), f16_cascades=[c for c in range(len(rays)) if (m >> c) & 1],
                         atlas_bytes=sum(n * (8 if (m >> c) & 1 else 16) for c, n in enumerate(rays)))
                 for k, m in rounded.items()}
        return {"scene": f"colonnade + {n_boxes} moving boxes: {s.triangle_count} triangles", "frames": frames,
                "dt_s": dt, "resolution": [width, height], "atlases": out, "shadow_map": shadow_size,
                "storage_rounding": {"modes": r_out, "rays_per_cascade": rays, "atlas_bytes_f32": 16 * sum(rays),
                                     "reference": "exact FP64 merge + SH + gather of the f32 trace; each mode rounds "
                                                  "the storage of its cascades to f16 with every stage in double"},
                "bricks_first_last": [c["bricks"] for c in counters],
                "error": "per valid pixel and rgb channel |x - x64| / max(|x64|, 1e-3 x frame mean |x64|); "
                         "quantiles are upper edges of 0.1-decade histogram bins"}
    finally:
        for rc in rcs.values():
            rc.destroy()
        if vox is not None:
            vox.destroy()
        sg.destroy()
