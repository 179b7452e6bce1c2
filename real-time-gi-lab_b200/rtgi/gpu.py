"""Host objects over the C-ABI: Context, SceneGpu (scene_gpu.ts uploadScene), VoxWorld (voxel.ts:710-727) and
Rc (rc.ts:980-992).  Method names follow the reference (update, encode, readCounters, usedBytes, readCounts,
setStats, destroy); errors raise GiError where the reference throws."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .configs import RcParams, VoxParams, cascade_layout, world_layout
from .scenes import Scene

_P = C.c_void_p


def _ptr(a: np.ndarray) -> int:
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def _stream(stream) -> Optional[int]:
    """A cudaStream_t from None, an int, or a torch.cuda.Stream."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


class Context:
    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = _P()
        _lib.call("gi_ctx_create", device, C.byref(h))
        self.handle = h
        self.device = device

    def destroy(self):
        if self.handle:
            _lib.call("gi_ctx_destroy", self.handle)
            self.handle = None


class SceneGpu:
    """uploadScene (scene_gpu.ts:56): vertices, triangle table and materials in device memory."""

    def __init__(self, ctx: Context, scene: Scene):
        self.ctx = ctx
        self.scene = scene
        pos = np.ascontiguousarray(scene.positions, dtype=np.float32)
        nrm = np.ascontiguousarray(scene.normals, dtype=np.float32)
        tri = np.ascontiguousarray(scene.tri, dtype=np.uint32)
        mats = scene.material_array()
        h = _P()
        _lib.call("gi_scene_upload", ctx.handle, _ptr(pos), _ptr(nrm), pos.shape[0], _ptr(tri), tri.shape[0],
                  _ptr(mats), len(mats), C.byref(h))
        self.handle = h
        if scene.textures is not None:
            self.set_textures(scene.textures, scene.uvs)

    def set_textures(self, images: np.ndarray, uvs: np.ndarray) -> None:
        """Base colour textures (gi_scene_set_textures): images (layers, size, size, 4) u8, uvs (V, 2) f32."""
        img = np.ascontiguousarray(images, dtype=np.uint8)
        uv = np.ascontiguousarray(uvs, dtype=np.float32)
        if img.ndim != 4 or img.shape[1] != img.shape[2] or img.shape[3] != 4:
            raise _lib.GiError(_lib.GI_ERR_INVALID, f"textures of shape {img.shape}: (layers, size, size, 4) expected")
        if uv.shape != (self.scene.positions.shape[0], 2):
            raise _lib.GiError(_lib.GI_ERR_INVALID, f"uvs of shape {uv.shape} for {self.scene.positions.shape[0]} vertices")
        _lib.call("gi_scene_set_textures", self.handle, _ptr(img), img.shape[1], img.shape[0], _ptr(uv))

    def set_draw_count(self, count: int) -> None:
        """The rasters draw rows [0, count) (a world's clustered copies are voxelised only)."""
        _lib.call("gi_scene_set_draw_count", self.handle, int(count))

    def set_static_count(self, count: int) -> None:
        """The voxel rebuild reads rows [0, count) (createVoxWorld's firstDynamicTri); the rest are dynamic."""
        _lib.call("gi_scene_set_static_count", self.handle, int(count))

    def set_draw_instances(self, offsets) -> None:
        """The rasters draw the drawn rows at every offset (instance 0 at the origin; None: once)."""
        if offsets is None or len(offsets) <= 1:
            _lib.call("gi_scene_set_draw_instances", self.handle, None, 1)
            return
        o = np.ascontiguousarray(np.asarray(offsets, np.float64).astype(np.float32).reshape(-1))
        _lib.call("gi_scene_set_draw_instances", self.handle, _ptr(o), len(offsets))

    def update_vertices(self, first: int, pos: np.ndarray, nrm: np.ndarray, stream=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        nrm = np.ascontiguousarray(nrm, dtype=np.float32)
        _lib.call("gi_scene_update_vertices", self.handle, first, pos.shape[0], _ptr(pos), _ptr(nrm), _stream(stream))

    def bytes(self) -> int:
        b = C.c_uint64()
        _lib.call("gi_scene_bytes", self.handle, C.byref(b))
        return b.value

    def rigid_define(self, first: int, verts_per_object: int, n_objects: int):
        """The vertex range [first, first + verts_per_object * n_objects) becomes rigid objects (rest = current)."""
        _lib.call("gi_scene_rigid_define", self.handle, first, verts_per_object, n_objects)

    def rigid_upload(self, m34, stream=None):
        """Row-major 3x4 transforms, one per object: a float32 array or a pointer to pinned host memory."""
        if isinstance(m34, np.ndarray):
            m34 = np.ascontiguousarray(m34, dtype=np.float32)
            _lib.call("gi_scene_rigid_upload", self.handle, _ptr(m34), _stream(stream))
        else:
            _lib.call("gi_scene_rigid_upload", self.handle, m34, _stream(stream))

    def rigid_apply(self, stream=None):
        _lib.call("gi_scene_rigid_apply", self.handle, _stream(stream))

    def set_raster_capacity(self, entries: int):
        """Entries of the G-buffer raster's per-tile lists (triangles past them are tested by every tile)."""
        _lib.call("gi_scene_set_raster_capacity", self.handle, entries)

    def destroy(self):
        if self.handle:
            _lib.call("gi_scene_destroy", self.handle)
            self.handle = None


class VoxWorld:
    """createVoxWorld (voxel.ts:746) / VoxWorld (voxel.ts:710-727)."""

    def __init__(self, scene: SceneGpu, params: VoxParams):
        self.scene = scene
        self.params = params
        p = _lib.GiVoxParams(float(params.v0), params.levels, params.G, params.maxBricks, params.maxVoxels,
                             params.dynBricks, 0)
        h = _P()
        _lib.call("gi_vox_create", scene.handle, C.byref(p), C.byref(h))
        self.handle = h

    def set_world(self, world) -> None:
        """Worlds (rtgi.world.World, the scene made by with_world): the instances and chunk lists; from the next update
        on the rebuild reads that frame's work items.  None: every row once."""
        self.world = world
        if world is None:
            _lib.call("gi_vox_set_world", self.handle, None, 0, None, 0, 0)
            return
        inst = np.ascontiguousarray(np.asarray(world.instances, np.float64).astype(np.float32).reshape(-1))
        lists = np.ascontiguousarray(world.lists(), np.uint32)
        _lib.call("gi_vox_set_world", self.handle, _ptr(inst), len(world.instances), _ptr(lists) if lists.size else None,
                  int(lists.size), int(world.rows))

    def update(self, eye) -> None:
        """writeUniform (voxel.ts:868-892): the windows around eye and, for a world, this frame's work items."""
        e = (C.c_double * 3)(*[float(x) for x in eye])
        _lib.call("gi_vox_update", self.handle, e)
        if getattr(self, "world", None) is not None:
            from . import world as W
            p = self.params
            rec, threads = W.item_records(W.select_items(self.world, W.windows(float(p.v0), p.levels, p.G, eye)))
            rec = np.ascontiguousarray(rec, np.uint32)
            _lib.call("gi_vox_set_items", self.handle, _ptr(rec) if len(rec) else None, len(rec), threads)

    def encode(self, stream=None, sun_rc=None) -> None:
        """The rebuild; with sun_rc, voxSun from that rc's shadow map and frame (gi_vox_build_sun)."""
        if sun_rc is not None:
            _lib.call("gi_vox_build_sun", self.handle, sun_rc.handle, _stream(stream))
        else:
            _lib.call("gi_vox_build", self.handle, _stream(stream))

    def read_counters(self, stream=None) -> dict:
        hdr = np.zeros(64, np.uint32)
        _lib.call("gi_vox_read_counters", self.handle, _ptr(hdr), _stream(stream))
        NL, mb = self.params.levels, self.params.maxBricks
        return {"bricks": int(min(hdr[0], mb)), "voxels": int(hdr[1]), "brickOverflow": int(hdr[2]),
                "bigOverflow": int(hdr[3]), "voxelOverflow": int(hdr[4]), "bricksPerLevel": [int(x) for x in hdr[8:8 + NL]],
                "bigPerLevel": [int(x) for x in hdr[16:16 + NL]], "hdr": hdr}

    def debug_hold_scan(self, part: int) -> None:
        """Test hook (gi_vox_debug_hold_scan): part `part` of the next rebuilds' brick scan publishes nothing, so the
        bounded wait after it gives up and read_counters raises GiError(GI_ERR_TIMEOUT); part < 0 turns it off."""
        _lib.call("gi_vox_debug_hold_scan", self.handle, int(part))

    def used_bytes(self) -> dict:
        a, b = C.c_uint64(), C.c_uint64()
        _lib.call("gi_vox_used_bytes", self.handle, C.byref(a), C.byref(b))
        return {"persistent": a.value, "buildTemp": b.value}

    def read_state(self, stream=None) -> dict:
        p = self.params
        per = p.G ** 3
        st = {"ptr": np.zeros(p.levels * per, np.uint32), "occ": np.zeros(p.maxBricks * 16, np.uint32),
              "base": np.zeros(p.maxBricks, np.uint32), "code": np.zeros(p.maxBricks, np.uint32),
              "rep": np.zeros(p.maxBricks * 512, np.uint32), "attr": np.zeros(p.maxVoxels * 4, np.uint32),
              "plane": np.zeros(p.maxVoxels, np.float32), "sunvis": np.zeros(p.maxVoxels, np.float32)}
        _lib.call("gi_vox_read_state", self.handle, *[_ptr(st[k]) for k in ("ptr", "occ", "base", "code", "rep", "attr", "plane", "sunvis")],
                  _stream(stream))
        st["hdr"] = self.read_counters(stream)["hdr"]
        return st

    def bytes(self) -> int:
        b = C.c_uint64()
        _lib.call("gi_vox_bytes", self.handle, C.byref(b))
        return b.value

    TUNING = ("chunk_cells", "blocks")

    def set_tuning(self, **kw):
        """Launch tuning of the rebuild (gi_vox_tuning): chunk_cells, blocks; unnamed fields keep their values."""
        cur = self.get_tuning()
        cur.update(kw)
        t = _lib.GiVoxTuning(*[cur[k] for k in self.TUNING])
        _lib.call("gi_vox_set_tuning", self.handle, C.byref(t))

    def get_tuning(self) -> dict:
        t = _lib.GiVoxTuning()
        _lib.call("gi_vox_get_tuning", self.handle, C.byref(t))
        return {k: int(getattr(t, k)) for k in self.TUNING}

    def destroy(self):
        if self.handle:
            _lib.call("gi_vox_destroy", self.handle)
            self.handle = None


ATLAS_CODES = {"f32": _lib.GI_ATLAS_F32, "f16": _lib.GI_ATLAS_F16, "bf16": _lib.GI_ATLAS_BF16}


class Rc:
    """createRc (rc.ts:1019) / Rc (rc.ts:980-992): screen or world probes, traced in the voxel world."""

    def __init__(self, ctx: Context, params: RcParams, width: int, height: int):
        if params.method not in ("screen", "world") or params.world != "voxel" or params.depthCascades != 0:
            raise _lib.GiError(_lib.GI_ERR_INVALID, f"unsupported configuration (method {params.method}, world "
                               f"{params.world}, depthCascades {params.depthCascades}): this library runs screen or "
                               "world probes traced in the voxel world (token 'voxel')")
        if params.cascades > 8:
            raise _lib.GiError(_lib.GI_ERR_INVALID, "at most 8 cascades")
        self.ctx, self.params, self.width, self.height = ctx, params, width, height
        self.world = params.method == "world"
        self.layout = world_layout(params) if self.world else cascade_layout(params, width, height)
        p = _lib.GiRcParams()
        p.cascades, p.P, p.k_interval = params.cascades, params.P, params.kInterval
        p.vox_scale, p.vox_offset, p.vox_skip, p.level_map = params.voxScale, params.voxOffset, params.voxSkip, params.levelMap
        p.res_cap, p.dda_cap, p.stats, p.atlas = params.resCap, params.ddaCap, params.stats, ATLAS_CODES[params.atlas]
        p.f32_out = 1 if params.f32Out else 0
        p.irr_f16 = 1 if params.irr16 else 0
        h = _P()
        if self.world:
            wp = _lib.GiWorldParams()
            wp.relocate = {"gbuffer": _lib.GI_RELOCATE_GBUFFER, "none": _lib.GI_RELOCATE_NONE,
                           "voxel": _lib.GI_RELOCATE_VOXEL}[params.relocate]
            for i in range(params.cascades):
                wp.caps[i] = int(params.caps[i])
            _lib.call("gi_rc_create_world", ctx.handle, C.byref(p), C.byref(wp), width, height, C.byref(h))
        else:
            _lib.call("gi_rc_create", ctx.handle, C.byref(p), width, height, C.byref(h))
        self.handle = h
        if params.objects:
            self.set_objects(True)

    def set_frame(self, frame: np.ndarray, stream=None):
        frame = np.ascontiguousarray(frame, dtype=np.float32)
        assert frame.size == 160
        _lib.call("gi_rc_set_frame", self.handle, _ptr(frame), _stream(stream))

    def set_gbuffer(self, depth: np.ndarray, normal: np.ndarray, stream=None):
        depth = np.ascontiguousarray(depth, dtype=np.float32)
        if normal.dtype == np.float16 or normal.dtype == np.uint16:
            n16 = np.ascontiguousarray(normal).view(np.uint16)
            _lib.call("gi_rc_set_gbuffer_f16", self.handle, _ptr(depth), _ptr(n16), _stream(stream))
        else:
            n32 = np.ascontiguousarray(normal, dtype=np.float32)
            _lib.call("gi_rc_set_gbuffer", self.handle, _ptr(depth), _ptr(n32), _stream(stream))

    def render_gbuffer(self, scene: SceneGpu, stream=None):
        _lib.call("gi_rc_render_gbuffer", self.handle, scene.handle, _stream(stream))

    def render_shadow(self, scene: SceneGpu, size: int = 4096, stream=None):
        """The sun shadow map from the frame's lightViewProj (encodeShadow, lighting.ts:175-189); while it is held,
        solves run voxSun with it.  size 0 releases it."""
        _lib.call("gi_rc_render_shadow", self.handle, scene.handle, int(size), _stream(stream))
        self.shadow_size = int(size)

    def set_bounce(self, vox: "VoxWorld", cell: float = 1.2, dims=(32, 16, 32), rays: int = 16, div: int = 2):
        """Multi-bounce (bounce.ts, DEFAULT_BOUNCE) bound to `vox`; vox None turns it off."""
        if vox is None:
            _lib.call("gi_rc_set_bounce", self.handle, None, None)
            return
        p = _lib.GiBounceParams(cell, dims[0], dims[1], dims[2], rays, div)
        _lib.call("gi_rc_set_bounce", self.handle, vox.handle, C.byref(p))

    def read_shadow(self, stream=None) -> np.ndarray:
        """The shadow map: (S, S), or (2, S, S) when drawn for a frame with two layers."""
        S = getattr(self, "shadow_size", 0)
        m = self.read_buffer(_lib.GI_RC_SHADOW, stream).view(np.float32).reshape(-1, S, S)
        return m[0] if m.shape[0] == 1 else m

    def encode(self, vox: VoxWorld, stream=None):
        _lib.call("gi_rc_solve", self.handle, vox.handle, _stream(stream))

    def solve(self, vox: VoxWorld, stream=None):
        """One frame of the GI path: the voxel rebuild, then the cascades."""
        _lib.call("gi_solve", self.handle, vox.handle, _stream(stream))

    def read_irradiance(self, stream=None) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        _lib.call("gi_rc_read_irradiance", self.handle, _ptr(out), _stream(stream))
        return out

    def read_counts(self, stream=None) -> np.ndarray:
        out = np.zeros(80, np.uint32)
        _lib.call("gi_rc_read_counts", self.handle, _ptr(out), _stream(stream))
        return out

    def set_stats(self, level: int):
        _lib.call("gi_rc_set_stats", self.handle, level)
        self.params.stats = level

    def set_dyn(self, dyn: Optional["DynLayer"]):
        """The dynamic layer the traces read (gi_rc_set_dyn); gi_solve builds it after the static rebuild."""
        _lib.call("gi_rc_set_dyn", self.handle, dyn.handle if dyn is not None else None)

    def set_objects(self, on: bool):
        """The token obj (phase 31): the bound layer's objects receive the bounce volume's light and block and
        reflect the volume's rays (gi_rc_set_objects); set from RcParams.objects at creation."""
        _lib.call("gi_rc_set_objects", self.handle, 1 if on else 0)

    def set_debug_hits(self, on: bool):
        _lib.call("gi_rc_set_debug_hits", self.handle, 1 if on else 0)

    def graph_capture(self, vox: VoxWorld, stream):
        """Captures one solve (voxel rebuild + cascades) into a CUDA graph owned by this Rc."""
        _lib.call("gi_rc_graph_capture", self.handle, vox.handle, _stream(stream))

    def graph_capture_frame(self, vox: VoxWorld, scene: SceneGpu, irr_ptr: Optional[int], stream):
        """Captures a whole frame: rigid pose, G-buffer, voxel rebuild, cascades, irradiance copy to irr_ptr."""
        _lib.call("gi_rc_graph_capture_frame", self.handle, vox.handle, scene.handle, irr_ptr, _stream(stream))

    def graph_launch(self, stream):
        _lib.call("gi_rc_graph_launch", self.handle, _stream(stream))

    def read_irradiance_raw(self, out: np.ndarray, stream=None):
        _lib.call("gi_rc_read_irradiance_raw", self.handle, out.ctypes.data if isinstance(out, np.ndarray) else out,
                  out.nbytes if isinstance(out, np.ndarray) else self.irr_bytes(), _stream(stream))

    def merge_gather_f64(self, stream=None, f16_cascades: int = 0):
        """FP64 reference of merge + SH + gather from the last trace (f32 atlas, debug hits on).  f16_cascades: bit
        mask of cascades whose atlas storage is rounded to f16 (traced intervals and, above cascade 0, merged
        radiances), every stage still in double."""
        if f16_cascades:
            _lib.call("gi_rc_merge_gather_f64_rounded", self.handle, int(f16_cascades), _stream(stream))
        else:
            _lib.call("gi_rc_merge_gather_f64", self.handle, _stream(stream))

    def read_irradiance_f64(self, ptr: Optional[int] = None, stream=None) -> Optional[np.ndarray]:
        """The FP64 irradiance, (H, W, 4) doubles; into the host or device memory at ptr when given."""
        if ptr is not None:
            _lib.call("gi_rc_read_irradiance_f64", self.handle, ptr, _stream(stream))
            return None
        out = np.zeros((self.height, self.width, 4), np.float64)
        _lib.call("gi_rc_read_irradiance_f64", self.handle, _ptr(out), _stream(stream))
        return out

    def read_irradiance_async(self, ptr: int, stream):
        """Stream-ordered copy of the stored irradiance into host or device memory at ptr (irr_bytes() bytes)."""
        _lib.call("gi_rc_read_irradiance_async", self.handle, ptr, self.irr_bytes(), _stream(stream))

    def irr_bytes(self) -> int:
        wide = (self.params.atlas == "f32" or self.params.f32Out) and not self.params.irr16
        return self.width * self.height * (16 if wide else 8)

    def set_gbuffer_tag(self, tag: np.ndarray, stream=None):
        """The G-buffer's style tags (H x W bytes, the albedo's alpha: 255 toon, 128 object, 0 photoreal)."""
        tag = np.ascontiguousarray(tag, dtype=np.uint8)
        if tag.size != self.width * self.height:
            raise _lib.GiError(_lib.GI_ERR_INVALID, f"tag of {tag.size} bytes for {self.width}x{self.height}")
        _lib.call("gi_rc_set_gbuffer_tag", self.handle, _ptr(tag), _stream(stream))

    def set_gbuffer_ptrs(self, depth_ptr: int, normal_f16_ptr: int, stream=None, rgb: bool = False):
        """G-buffer from host pointers (pinned memory makes the copies asynchronous); rgb: the normals as three
        halves per pixel (gi_rc_set_gbuffer_rgb16f) instead of four."""
        _lib.call("gi_rc_set_gbuffer_rgb16f" if rgb else "gi_rc_set_gbuffer_f16", self.handle, depth_ptr,
                  normal_f16_ptr, _stream(stream))

    def set_frame_ptr(self, frame_ptr: int, stream=None):
        _lib.call("gi_rc_set_frame", self.handle, frame_ptr, _stream(stream))

    def read_irradiance_raw_ptr(self, ptr: int, stream=None):
        _lib.call("gi_rc_read_irradiance_raw", self.handle, ptr, self.irr_bytes(), _stream(stream))

    PASSES = ("vox", "giBuild", "giTrace", "giMerge", "giGather")
    TUNING = ("trace_order", "trace_rays", "trace_blocks", "gather_shape", "merge_threads")

    def set_tuning(self, **kw):
        """Launch tuning of the cascade passes (gi_rc_tuning); unnamed fields keep their values."""
        cur = self.get_tuning()
        cur.update(kw)
        t = _lib.GiRcTuning(*[cur[k] for k in self.TUNING])
        _lib.call("gi_rc_set_tuning", self.handle, C.byref(t))

    def get_tuning(self) -> dict:
        t = _lib.GiRcTuning()
        _lib.call("gi_rc_get_tuning", self.handle, C.byref(t))
        return {k: int(getattr(t, k)) for k in self.TUNING}

    def set_timing(self, on: bool):
        _lib.call("gi_rc_set_timing", self.handle, 1 if on else 0)

    def pass_times(self) -> dict:
        ms = np.zeros(5, np.float32)
        _lib.call("gi_rc_pass_times", self.handle, _ptr(ms))
        return dict(zip(self.PASSES, [float(x) for x in ms]))

    def bytes(self) -> int:
        b = C.c_uint64()
        _lib.call("gi_rc_bytes", self.handle, C.byref(b))
        return b.value

    def read_buffer(self, what: int, stream=None) -> np.ndarray:
        n = C.c_size_t()
        _lib.call("gi_rc_buffer_bytes", self.handle, what, C.byref(n))
        out = np.zeros(n.value, np.uint8)
        _lib.call("gi_rc_read_buffer", self.handle, what, _ptr(out), n.value, _stream(stream))
        return out

    def read_atlas(self, what: int = _lib.GI_RC_RAD, stream=None) -> np.ndarray:
        """The atlas (or SH) as f32 values, (n, 4)."""
        raw = self.read_buffer(what, stream)
        if self.params.atlas == "f32" or (what == _lib.GI_RC_SH and self.params.f32Out):
            return raw.view(np.float32).reshape(-1, 4)
        if self.params.atlas == "f16":
            return raw.view(np.float16).astype(np.float32).reshape(-1, 4)
        return (raw.view(np.uint16).astype(np.uint32) << 16).view(np.float32).reshape(-1, 4)

    def read_world(self, stream=None) -> dict:
        """World probes: the hash tables, their slots' probes, the parents and the state words."""
        u = lambda what: self.read_buffer(what, stream).view(np.uint32)
        return {"keys": u(_lib.GI_RC_WORLD_KEYS), "slot_probe": u(_lib.GI_RC_WORLD_SLOTS),
                "parents": u(_lib.GI_RC_WORLD_PARENTS), "state": u(_lib.GI_RC_WORLD_STATE)}

    def destroy(self):
        if self.handle:
            _lib.call("gi_rc_destroy", self.handle)
            self.handle = None


class DynLayer:
    """The dynamic layer (dynlayer.ts createDynLayer / DynLayer) of a voxel world: its scene's rows from first_dynamic
    on, splatted every build; bind it to an Rc (Rc.set_dyn) for its traces to read it."""

    def __init__(self, vox: VoxWorld, first_dynamic: int, bricks: int = 512, albedo: bool = False):
        h = C.c_void_p()
        _lib.call("gi_dyn_create", vox.handle, bricks, first_dynamic, 1 if albedo else 0, C.byref(h))
        self.handle, self.vox, self.bricks = h, vox, bricks

    def build(self, rc: "Rc", stream=None) -> None:
        _lib.call("gi_dyn_build", self.handle, rc.handle, _stream(stream))

    def read_counters(self, stream=None) -> dict:
        hdr = np.zeros(64, np.uint32)
        _lib.call("gi_dyn_read_counters", self.handle, _ptr(hdr), _stream(stream))
        return {"bricks": int(hdr[8]), "brickOverflow": int(hdr[1]), "outside": int(hdr[9]), "hdr": hdr}

    def read_state(self, stream=None) -> dict:
        p = self.vox.params
        nptr = p.levels * p.G ** 3
        st = {"ptr": np.zeros(nptr, np.uint32), "bits": np.zeros(2 * nptr // 32, np.uint32),
              "meta": np.zeros(self.bricks, np.uint32), "mask": np.zeros(self.bricks * 16, np.uint32),
              "data": np.zeros(self.bricks * 512 * 13, np.uint32)}
        _lib.call("gi_dyn_read_state", self.handle, *[_ptr(st[k]) for k in ("ptr", "bits", "meta", "mask", "data")],
                  _stream(stream))
        st["hdr"] = self.read_counters(stream)["hdr"]
        return st

    def destroy(self):
        if self.handle:
            _lib.call("gi_dyn_destroy", self.handle)
            self.handle = None


class Batch:
    """n independent solves captured into one CUDA graph (gi_batch_*): parallel solve chains (capture), or the
    rebuilds in parallel then one launch per cascade pass over every solve (capture_passes)."""

    def __init__(self, ctx: Context, rcs, voxes):
        assert len(rcs) == len(voxes)
        self.ctx, self.rcs, self.voxes = ctx, list(rcs), list(voxes)
        n = len(rcs)
        ra = (_P * n)(*[r.handle for r in rcs])
        va = (_P * n)(*[v.handle for v in voxes])
        h = _P()
        _lib.call("gi_batch_create", ctx.handle, ra, va, n, C.byref(h))
        self.handle = h

    def capture(self, stream):
        _lib.call("gi_batch_capture", self.handle, _stream(stream))

    def capture_passes(self, stream):
        """The rebuilds as parallel branches, then one launch per cascade pass over every solve."""
        _lib.call("gi_batch_capture_passes", self.handle, _stream(stream))

    def launch(self, stream):
        _lib.call("gi_batch_launch", self.handle, _stream(stream))

    def destroy(self):
        if self.handle:
            _lib.call("gi_batch_destroy", self.handle)
            self.handle = None
