"""Parameters and the config-name grammar (src/core/rc.ts:42-91 RcParams / DEFAULT_PARAMS, src/core/voxel.ts:31-50
VoxParams / DEFAULT_VOX / voxParams, src/runner/configs.ts:47-73 parseConfig).

Same names, defaults and error behaviour: unknown config tokens and unknown voxel parameters raise.  This build adds
five RcParams fields and their tokens: ``ddaCap`` (token ``dda<N>``; the reference hard-codes 1024 steps,
voxel.ts:142), ``atlas`` (tokens ``f32``/``f16``/``bf16``; the reference stores f16), ``f32Out`` (token ``f32out``:
SH and irradiance kept in f32 whatever the atlas), ``irr16`` (token ``irr16``: the irradiance stored as rgba16float,
the reference's rc.irr format, whatever the atlas; the passes before the store keep their precision) and ``stats``.
"""
from __future__ import annotations

import dataclasses
import re
from dataclasses import dataclass, field
from typing import List, Optional


@dataclass
class RcParams:
    method: str = "world"
    P: int = 8
    cascades: int = 5
    sMin: float = 0.05
    kInterval: float = 1.0
    regStride: int = 1
    rayStride: int = 1
    maxSteps: int = 16
    pxStride: float = 4
    thicknessMin: float = 0.15
    lift: float = 0.25
    caps: List[int] = field(default_factory=lambda: [1 << 18, 1 << 16, 1 << 14, 1 << 12, 1 << 11, 1 << 10, 1 << 9, 1 << 8])
    analytic: bool = False
    world: str = "none"
    depthCascades: int = 8
    levelMap: float = 1
    voxScale: float = 0.25
    voxOffset: float = 1
    voxSkip: float = 0.5
    resCap: int = 8
    stats: int = 0
    relocate: str = "gbuffer"
    styleEmit: bool = True
    styleRecv: bool = True
    rampSoft: float = 0
    ddgi: Optional[dict] = None
    bounce: bool = True
    objects: bool = False
    gl2: Optional[dict] = None
    # additions of this build
    ddaCap: int = 1024
    atlas: str = "f16"
    f32Out: bool = False
    irr16: bool = False


DEFAULT_PARAMS = RcParams()


def parse_config(name: str, overrides: Optional[dict] = None) -> RcParams:
    """parseConfig (configs.ts:47-73): `<method>-<P>[-token...]`."""
    overrides = dict(overrides or {})
    if name.startswith("ddgi-") or name.startswith("gl2-"):
        raise ValueError(f"{name}: the DDGI and WebGL2 comparators are not part of this library")
    method, P, *tokens = name.split("-")
    p = dataclasses.replace(DEFAULT_PARAMS, **overrides)
    p.method, p.P = method, int(P)
    for t in tokens:
        if t == "analytic": p.analytic = True
        elif t == "depth": p.world = "none"
        elif t == "voxel": p.world, p.depthCascades = "voxel", 0
        elif t == "hybrid": p.world, p.depthCascades = "voxel", 1
        elif t == "tri": p.world, p.depthCascades = "tri", 0
        elif t == "trihybrid": p.world, p.depthCascades = "tri", 1
        elif t == "l2": p.levelMap = 2
        elif t == "norel": p.relocate = "none"
        elif t == "vrel": p.relocate = "voxel"
        elif t == "noemit": p.styleEmit = False
        elif t == "norecv": p.styleRecv = False
        elif re.fullmatch(r"soft[\d.]+", t): p.rampSoft = float(t[4:])
        elif re.fullmatch(r"rc\d", t): p.resCap = int(t[2:])
        elif re.fullmatch(r"vs[\d.]+", t): p.voxScale = float(t[2:])
        elif re.fullmatch(r"vo[\d.]+", t): p.voxOffset = float(t[2:])
        elif re.fullmatch(r"vk[\d.]+", t): p.voxSkip = float(t[2:])
        elif t == "obj": p.objects = True
        elif re.fullmatch(r"dda\d+", t): p.ddaCap = int(t[3:])
        elif t in ("f32", "f16", "bf16"): p.atlas = t
        elif t == "f32out": p.f32Out = True
        elif t == "irr16": p.irr16 = True
        else: raise ValueError(f"unknown config token {t} in {name}")
    return p


@dataclass
class VoxParams:
    v0: float = 0.2
    levels: int = 5
    G: int = 32
    maxBricks: int = 4608
    maxVoxels: int = 524288
    dynBricks: int = 512


DEFAULT_VOX = VoxParams()


def vox_params(o: Optional[dict] = None) -> VoxParams:
    """voxParams (voxel.ts:47-50): DEFAULT_VOX overridden; unknown keys raise."""
    o = dict(o or {})
    for k in o:
        if not hasattr(DEFAULT_VOX, k):
            raise ValueError(f"unknown voxel parameter {k}")
    return dataclasses.replace(DEFAULT_VOX, **o)


def cascade_layout(p: RcParams, width: int, height: int) -> dict:
    """The screen-method cascade layout (rc.ts:1027-1035): per cascade res = 4 << min(i, resCap), tile P << i,
    tiles = ceil(size / tile), interval [b_i, b_{i+1}] with b_k = kInterval (4^k - 1) / 3 (f64, stored f32)."""
    import numpy as np
    casc = []
    probe_off = rad_off = 0
    for i in range(p.cascades):
        res = 4 << min(i, p.resCap)
        ts = p.P << i
        tx, ty = -(-width // ts), -(-height // ts)
        b = lambda k: p.kInterval * (4 ** k - 1) / 3
        casc.append({"probe_off": probe_off, "cap": tx * ty, "rad_off": rad_off, "res": res, "tile_size": ts,
                     "tiles_x": tx, "tiles_y": ty, "b0": float(np.float32(b(i))), "b1": float(np.float32(b(i + 1)))})
        probe_off += tx * ty
        rad_off += tx * ty * res * res
    atlas = {"f32": 0, "f16": 1, "bf16": 2}[p.atlas]
    return {"cascades": p.cascades, "casc": casc, "vox_scale": p.voxScale, "vox_offset": p.voxOffset,
            "level_map": p.levelMap, "vox_skip": p.voxSkip, "dda_cap": p.ddaCap, "stats": p.stats, "atlas": atlas,
            "f32_out": 1 if p.f32Out else 0, "irr_f16": 1 if p.irr16 else 0,
            "probes_total": probe_off, "rays_total": rad_off}


def world_layout(p: RcParams) -> dict:
    """The world-method cascade layout (rc.ts:1027-1035): per cascade res = 4 << min(i, resCap), capacity caps[i],
    a hash table of nextPow2(2 cap) slots, interval [b_i, b_{i+1}]; probes and atlas entries by capacity."""
    import numpy as np
    casc = []
    probe_off = rad_off = hash_off = 0
    for i in range(p.cascades):
        res = 4 << min(i, p.resCap)
        cap = int(p.caps[i])
        if cap < 1:
            raise ValueError(f"cascade {i}: capacity {cap}")
        hs = 1 << max(0, (2 * cap - 1).bit_length())
        b = lambda k: p.kInterval * (4 ** k - 1) / 3
        casc.append({"probe_off": probe_off, "cap": cap, "rad_off": rad_off, "res": res, "tile_size": 0,
                     "tiles_x": 0, "tiles_y": 0, "hash_off": hash_off, "hash_mask": hs - 1,
                     "b0": float(np.float32(b(i))), "b1": float(np.float32(b(i + 1)))})
        probe_off += cap
        rad_off += cap * res * res
        hash_off += hs
    atlas = {"f32": 0, "f16": 1, "bf16": 2}[p.atlas]
    relocate = {"gbuffer": 0, "none": 1, "voxel": 2}[p.relocate]
    return {"cascades": p.cascades, "casc": casc, "vox_scale": p.voxScale, "vox_offset": p.voxOffset,
            "level_map": p.levelMap, "vox_skip": p.voxSkip, "dda_cap": p.ddaCap, "stats": p.stats, "atlas": atlas,
            "f32_out": 1 if p.f32Out else 0, "irr_f16": 1 if p.irr16 else 0, "probes_total": probe_off,
            "rays_total": rad_off,
            "hash_total": hash_off, "relocate": relocate, "world": True}
