"""ctypes binding of the oracle (oracle/_build/libgi_oracle.so).  Test infrastructure only: imported by tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the product path.

``build()`` compiles the oracle with its Makefile when the library is missing or older than its sources.
"""
from __future__ import annotations

import ctypes as C
import ctypes.util
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgi_oracle.so")
SOURCES = ["builtins.c", "vox.c", "rc.c", "rc64.c", "raster.c", "shadow.c", "world.c", "dyn.c", "tex.c", "orc_par.c", "gi_oracle.h", "orc_math.h",
           "orc_par.h", "orc_rc.h", "Makefile"]


def build(force: bool = False) -> str:
    newest = max(os.path.getmtime(os.path.join(HERE, s)) for s in SOURCES)
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_vox_build.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_rc_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_world_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_hash32.argtypes = [C.c_uint32]
        _lib.orc_hash32.restype = C.c_uint32
        _lib.orc_lod_for.argtypes = [C.c_void_p, C.c_float]
        _lib.orc_lod_for.restype = C.c_int32
        _lib.orc_rc_merge_gather.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_rc_merge_gather_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_rc_merge_gather_f64_rounded.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                                         C.c_void_p]
        _lib.orc_raster_gbuffer.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_pack4x8unorm.argtypes = [C.c_void_p]
        _lib.orc_pack4x8unorm.restype = C.c_uint32
        _lib.orc_pack2x16snorm.argtypes = [C.c_float, C.c_float]
        _lib.orc_pack2x16snorm.restype = C.c_uint32
        _lib.orc_f32_to_f16.argtypes = [C.c_float]
        _lib.orc_f32_to_f16.restype = C.c_uint16
        _lib.orc_f16_to_f32.argtypes = [C.c_uint16]
        _lib.orc_f16_to_f32.restype = C.c_float
        _lib.orc_f32_to_bf16.argtypes = [C.c_float]
        _lib.orc_f32_to_bf16.restype = C.c_uint16
        _lib.orc_tri_box.argtypes = [C.c_void_p] * 5
        _lib.orc_tri_box.restype = C.c_int
        _lib.orc_round_log2.argtypes = [C.c_float]
        _lib.orc_round_log2.restype = C.c_uint32
        _lib.orc_shadow_render.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        _lib.orc_sun_tap.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        _lib.orc_sun_tap.restype = C.c_float
        _lib.orc_tex_levels.argtypes = [C.c_uint32, C.c_void_p]
        _lib.orc_tex_levels.restype = C.c_uint32
        _lib.orc_tex_build.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        _lib.orc_tex_sample.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.c_void_p]
        _lib.orc_shadow_layers.argtypes = [C.c_void_p]
        _lib.orc_shadow_layers.restype = C.c_uint32
        _lib.orc_vox_sun.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        _lib.orc_bounce_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_gi_exp.argtypes = [C.c_float]
        _lib.orc_gi_exp.restype = C.c_float
        _lib.orc_dyn_init.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_dyn_build.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                       C.c_uint32]
        _lib.orc_trace_dyn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_void_p]
        _lib.orc_log2.argtypes = [C.c_float]
        _lib.orc_log2.restype = C.c_float
    return _lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class OrcScene(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("nrm", C.c_void_p), ("nverts", C.c_uint32), ("tri", C.c_void_p),
                ("ntris", C.c_uint32), ("mats", C.c_void_p), ("nmats", C.c_uint32),
                ("items", C.c_void_p), ("nitems", C.c_uint32), ("threads", C.c_uint32), ("key_stride", C.c_uint32),
                ("ninst", C.c_uint32), ("lists", C.c_void_p), ("inst", C.c_void_p),
                ("ndraw", C.c_uint32), ("draw_ninst", C.c_uint32), ("draw_inst", C.c_void_p),
                ("uv", C.c_void_p), ("tex", C.c_void_p), ("tex_size", C.c_uint32), ("tex_levels", C.c_uint32),
                ("tex_layers", C.c_uint32), ("tex_layer_texels", C.c_uint32)]


class OrcVox(C.Structure):
    _fields_ = [("v0", C.c_float), ("levels", C.c_uint32), ("G", C.c_uint32), ("max_bricks", C.c_uint32),
                ("max_voxels", C.c_uint32), ("big_cap", C.c_uint32), ("coarse_from_triangles", C.c_uint32),
                ("origin", (C.c_int32 * 4) * 8),
                ("hdr", C.c_void_p), ("ptr", C.c_void_p), ("occ", C.c_void_p), ("base", C.c_void_p),
                ("code", C.c_void_p), ("rep", C.c_void_p), ("big", C.c_void_p), ("attr", C.c_void_p),
                ("plane", C.c_void_p), ("sunvis", C.c_void_p), ("bn_inj", C.c_void_p), ("dyn", C.c_void_p)]


class OrcDyn(C.Structure):
    _fields_ = [("nb", C.c_uint32), ("albedo", C.c_uint32), ("hdr", C.c_void_p), ("ptr", C.c_void_p),
                ("bits", C.c_void_p), ("meta", C.c_void_p), ("mask", C.c_void_p), ("data", C.c_void_p)]


class OrcBounce(C.Structure):
    _fields_ = [("cell", C.c_float), ("v0", C.c_float), ("dx", C.c_uint32), ("dy", C.c_uint32), ("dz", C.c_uint32),
                ("rays", C.c_uint32), ("div", C.c_uint32), ("dirs", C.c_void_p), ("vol", C.c_void_p * 2),
                ("list", C.c_void_p), ("objects", C.c_uint32)]


class OrcCasc(C.Structure):
    _fields_ = [("probe_off", C.c_uint32), ("cap", C.c_uint32), ("rad_off", C.c_uint32), ("res", C.c_uint32),
                ("tile_size", C.c_uint32), ("tiles_x", C.c_uint32), ("tiles_y", C.c_uint32), ("pad", C.c_uint32),
                ("b0", C.c_float), ("b1", C.c_float), ("pad2", C.c_float * 2)]


class OrcLayout(C.Structure):
    _fields_ = [("cascades", C.c_uint32), ("c", OrcCasc * 8), ("vox_scale", C.c_float), ("vox_offset", C.c_float),
                ("level_map", C.c_float), ("vox_skip", C.c_float), ("dda_cap", C.c_uint32), ("stats", C.c_uint32),
                ("atlas", C.c_uint32), ("f32_out", C.c_uint32), ("irr_f16", C.c_uint32)]


class OrcGbuf(C.Structure):
    _fields_ = [("frame", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32), ("depth", C.c_void_p),
                ("normal", C.c_void_p), ("tag", C.c_void_p)]


class OrcRcOut(C.Structure):
    _fields_ = [("probes", C.c_void_p), ("rad", C.c_void_p), ("sh", C.c_void_p), ("irr", C.c_void_p),
                ("counts", C.c_void_p), ("hit", C.c_void_p)]


class OrcWLayout(C.Structure):
    _fields_ = [("base", OrcLayout), ("hash_off", C.c_uint32 * 8), ("hash_mask", C.c_uint32 * 8),
                ("hash_total", C.c_uint32), ("relocate", C.c_uint32)]


class OrcWState(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("slot_probe", C.c_void_p), ("parents", C.c_void_p), ("hist_tab", C.c_void_p),
                ("hist_grid", C.c_void_p), ("hist_sh", C.c_void_p), ("hist_par", C.c_uint32)]


PROBE_DTYPE = np.dtype([("pos", "<f4", (4,)), ("nrm", "<f4", (4,)), ("grid", "<i4", (4,))])


def _scene_struct(scene):
    pos = np.ascontiguousarray(scene.positions, dtype=np.float32)
    nrm = np.ascontiguousarray(scene.normals, dtype=np.float32)
    tri = np.ascontiguousarray(scene.tri, dtype=np.uint32)
    mats = scene.material_array()
    s = OrcScene(_p(pos), _p(nrm), pos.shape[0], _p(tri), tri.shape[0], _p(mats), len(mats))
    keep = [pos, nrm, tri, mats]
    if getattr(scene, "textures", None) is not None:
        img = np.ascontiguousarray(scene.textures, dtype=np.uint8)
        uv = np.ascontiguousarray(scene.uvs, dtype=np.float32)
        tex = texture_chain(img)
        size, layers = img.shape[1], img.shape[0]
        per = C.c_uint32(0)
        levels = lib().orc_tex_levels(size, C.byref(per))
        s.uv, s.tex, s.tex_size, s.tex_levels, s.tex_layers, s.tex_layer_texels = \
            _p(uv), _p(tex), size, levels, layers, per.value
        keep += [uv, tex]
    return s, tuple(keep)


def tex_sample(img: np.ndarray, u: float, v: float, lod: int, layer: int = 1) -> np.ndarray:
    """One sample of the oracle's texture definition (orc_tex_sample) from images (layers, size, size, 4) u8."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    tex = texture_chain(img)
    per = C.c_uint32(0)
    levels = lib().orc_tex_levels(img.shape[1], C.byref(per))
    s = OrcScene()
    uv = np.zeros(2, np.float32)
    s.uv, s.tex, s.tex_size, s.tex_levels, s.tex_layers, s.tex_layer_texels = \
        _p(uv), _p(tex), img.shape[1], levels, img.shape[0], per.value
    out = np.zeros(4, np.float32)
    lib().orc_tex_sample(C.byref(s), layer, C.c_float(u), C.c_float(v), lod, _p(out))
    return out


_TEX_CACHE = {}


def texture_chain(img: np.ndarray) -> np.ndarray:
    """The decoded layers and their mip chains (orc_tex_build), cached per image content."""
    key = (img.shape, hash(img.tobytes()))
    hit = _TEX_CACHE.get(key)
    if hit is not None:
        return hit
    per = C.c_uint32(0)
    lib().orc_tex_levels(img.shape[1], C.byref(per))
    out = np.zeros((img.shape[0], per.value, 4), np.float32)
    lib().orc_tex_build(_p(img), img.shape[1], img.shape[0], _p(out))
    _TEX_CACHE.clear()
    _TEX_CACHE[key] = out
    return out


def vox_origins(v0: float, levels: int, G: int, eye) -> np.ndarray:
    """writeUniform's per-level window origins (voxel.ts:872-876), host f64 math."""
    import math
    o = np.zeros((8, 4), dtype=np.int32)
    for L in range(levels):
        bs = v0 * 2 ** L * 8
        for a in range(3):
            o[L, a] = math.floor(eye[a] / bs) - G // 2
    return o


def vox_build(scene, v0: float, levels: int, G: int, max_bricks: int, max_voxels: int, eye,
              coarse_from_triangles: bool = False, big_cap: int = 1 << 18, world=None) -> dict:
    """The rebuild; with `world` (rtgi.world.World, the scene its with_world output) the work items of the windows
    around eye (selectItems) instead of every row."""
    s, keep = _scene_struct(scene)
    if world is not None:
        from rtgi import world as W
        items, threads = W.item_records(W.select_items(world, W.windows(float(v0), levels, G, eye)))
        lists = world.lists()
        inst = np.zeros((len(world.instances), 4), np.float32)
        inst[:, :3] = np.asarray(world.instances, np.float64).astype(np.float32)
        nitems = len(items)
        items = np.ascontiguousarray(items if nitems else np.zeros((1, 4), np.uint32), np.uint32)
        lists = np.ascontiguousarray(lists if lists.size else np.zeros(1, np.uint32), np.uint32)
        keep = keep + (items, lists, inst)
        s.items, s.nitems, s.threads = _p(items), nitems, threads
        s.key_stride, s.ninst, s.lists, s.inst = world.rows, len(world.instances), _p(lists), _p(inst)
    per = G ** 3
    st = {
        "hdr": np.zeros(64, np.uint32), "ptr": np.zeros(levels * per, np.uint32),
        "occ": np.zeros(max_bricks * 16, np.uint32), "base": np.zeros(max_bricks, np.uint32),
        "code": np.zeros(max_bricks, np.uint32), "rep": np.zeros(max_bricks * 512, np.uint32),
        "big": np.zeros(16 * big_cap, np.uint32), "attr": np.zeros(max_voxels * 4, np.uint32),
        "plane": np.zeros(max_voxels, np.float32), "sunvis": np.zeros(max_voxels, np.float32),
    }
    vx = OrcVox()
    vx.v0 = np.float32(v0)
    vx.levels, vx.G, vx.max_bricks, vx.max_voxels, vx.big_cap = levels, G, max_bricks, max_voxels, big_cap
    vx.coarse_from_triangles = 1 if coarse_from_triangles else 0
    org = vox_origins(float(v0), levels, G, eye)   # f64 v0, as the reference's numbers (voxel.ts:873)
    for L in range(8):
        for a in range(4):
            vx.origin[L][a] = int(org[L, a])
    for k in ("hdr", "ptr", "occ", "base", "code", "rep", "big", "attr", "plane", "sunvis"):
        setattr(vx, k, _p(st[k]))
    lib().orc_vox_build(C.byref(s), C.byref(vx))
    del st["big"]
    st.update(v0=float(np.float32(v0)), levels=levels, G=G, max_bricks=max_bricks, max_voxels=max_voxels, origin=org)
    return st


def _vox_struct(st: dict) -> OrcVox:
    vx = OrcVox()
    vx.v0 = st["v0"]
    vx.levels, vx.G, vx.max_bricks, vx.max_voxels = st["levels"], st["G"], st["max_bricks"], st["max_voxels"]
    vx.big_cap = 0
    for L in range(8):
        for a in range(4):
            vx.origin[L][a] = int(st["origin"][L, a])
    for k in ("hdr", "ptr", "occ", "base", "code", "rep", "attr", "plane", "sunvis"):
        setattr(vx, k, _p(st[k]))
    vx.big = None
    vx.bn_inj = _p(st["bn_inj"]) if st.get("bn_inj") is not None else None
    vx.dyn = C.addressof(st["dyn"].struct) if st.get("dyn") is not None else None
    return vx


def layout_struct(lay: dict) -> OrcLayout:
    ly = OrcLayout()
    ly.cascades = lay["cascades"]
    for i, c in enumerate(lay["casc"]):
        ly.c[i].probe_off, ly.c[i].cap, ly.c[i].rad_off, ly.c[i].res = c["probe_off"], c["cap"], c["rad_off"], c["res"]
        ly.c[i].tile_size, ly.c[i].tiles_x, ly.c[i].tiles_y = c["tile_size"], c["tiles_x"], c["tiles_y"]
        ly.c[i].b0, ly.c[i].b1 = c["b0"], c["b1"]
    ly.vox_scale, ly.vox_offset, ly.level_map, ly.vox_skip = lay["vox_scale"], lay["vox_offset"], lay["level_map"], lay["vox_skip"]
    ly.dda_cap, ly.stats, ly.atlas = lay["dda_cap"], lay["stats"], lay["atlas"]
    ly.f32_out = lay.get("f32_out", 0)
    ly.irr_f16 = lay.get("irr_f16", 0)
    return ly


def rc_solve(vox: dict, lay: dict, frame: np.ndarray, depth: np.ndarray, normal: np.ndarray, want_hit: bool = False,
             merge: bool = True) -> dict:
    """setupScreen + trace, then (merge=True) mergeScreen + projectSH + gatherScreen.  Returns numpy outputs; 'rad_traced'
    is the atlas right after the trace."""
    H, W = depth.shape
    ly = layout_struct(lay)
    probes_total = sum(c["cap"] for c in lay["casc"])
    rad_total = sum(c["cap"] * c["res"] ** 2 for c in lay["casc"])
    out = {"probes": np.zeros(probes_total, PROBE_DTYPE), "rad": np.zeros((rad_total, 4), np.float32),
           "sh": np.zeros((lay["casc"][0]["cap"], 32), np.float32), "irr": np.zeros((H, W, 4), np.float32),
           "counts": np.zeros(80, np.uint32)}
    if want_hit:
        out["hit"] = np.zeros((rad_total, 4), np.uint32)
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    normal = np.ascontiguousarray(normal, dtype=np.float32)
    g = OrcGbuf(_p(frame), W, H, _p(depth), _p(normal), None)
    o = OrcRcOut(_p(out["probes"]), _p(out["rad"]), _p(out["sh"]), _p(out["irr"]), _p(out["counts"]),
                 _p(out["hit"]) if want_hit else None)
    vx = _vox_struct(vox)
    lib().orc_rc_trace(C.byref(vx), C.byref(ly), C.byref(g), C.byref(o))
    out["rad_traced"] = out["rad"].copy()
    if merge:
        lib().orc_rc_merge_gather(C.byref(ly), C.byref(g), C.byref(o))
    return out


def merge_gather_f64(lay: dict, frame: np.ndarray, depth: np.ndarray, normal: np.ndarray, probes: np.ndarray,
                     rad_traced: np.ndarray, f16_cascades: int = 0) -> np.ndarray:
    """FP64 merge + SH + gather of the traced intervals; f16_cascades: cascades whose atlas storage is rounded to f16."""
    H, W = depth.shape
    ly = layout_struct(lay)
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    normal = np.ascontiguousarray(normal, dtype=np.float32)
    probes = np.ascontiguousarray(probes)
    rad = np.ascontiguousarray(rad_traced, dtype=np.float32)
    irr = np.zeros((H, W, 4), np.float64)
    g = OrcGbuf(_p(frame), W, H, _p(depth), _p(normal), None)
    lib().orc_rc_merge_gather_f64_rounded(C.byref(ly), C.byref(g), _p(probes), _p(rad), int(f16_cascades), _p(irr))
    return irr


def _drawn(s, keep, ndraw, draw_instances):
    """The rasters' drawn rows and instances (instance 0 at the origin)."""
    s.ndraw = int(ndraw)
    if draw_instances is not None and len(draw_instances) > 1:
        inst = np.zeros((len(draw_instances), 4), np.float32)
        inst[:, :3] = np.asarray(draw_instances, np.float64).astype(np.float32)
        s.draw_inst, s.draw_ninst = _p(inst), len(draw_instances)
        keep = keep + (inst,)
    return keep


def raster_gbuffer(scene, frame: np.ndarray, W: int, H: int, ndraw: int = 0, draw_instances=None):
    """The G-buffer of rows [0, ndraw) (0: every row) at every draw instance."""
    s, keep = _scene_struct(scene)
    keep = _drawn(s, keep, ndraw, draw_instances)
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    depth = np.zeros((H, W), np.float32)
    normal = np.zeros((H, W, 4), np.float32)
    tri = np.zeros((H, W), np.uint32)
    r = lib().orc_raster_gbuffer(C.byref(s), _p(frame), W, H, _p(depth), _p(normal), _p(tri))
    if r != 0:
        raise MemoryError("oracle raster: out of memory")
    return depth, normal, tri


def toon_receive(c, n, soft: float) -> np.ndarray:
    """toonReceive of (c0, c1y, c1z, c1x) (12 floats) for normal n: (E rgb, band, contrast)."""
    c = np.ascontiguousarray(c, np.float32)
    n = np.ascontiguousarray(n, np.float32)
    out = np.zeros(5, np.float32)
    lib().orc_toon_receive(_p(c), _p(n), C.c_float(soft), _p(out))
    return out


def gbuffer_tags(scene, tri: np.ndarray, ndraw: int = 0) -> np.ndarray:
    """The G-buffer's style tags (gbuffer.ts:2, the albedo's alpha byte) from the raster's triangle per pixel
    (instance * ndraw + row; 0xffffffff: background): 255 for a toon material (flag 4), 128 for another measured
    object (flag 8), 0 for photoreal materials and the background."""
    flags = np.array([int(m.flags) for m in scene.materials], np.uint32)
    t = np.asarray(tri, np.int64)
    bg = t == 0xffffffff
    row = np.where(bg, 0, t % (ndraw or scene.triangle_count))
    f = np.where(bg, 0, flags[np.asarray(scene.tri, np.int64)[row, 3]])
    return np.where(f & 4, 255, np.where(f & 8, 128, 0)).astype(np.uint8)


def shadow_render(scene, frame: np.ndarray, S: int, ndraw: int = 0, draw_instances=None) -> np.ndarray:
    """The sun shadow map (S x S depths, 1 = nothing drawn) from the frame's lightViewProj; (2, S, S) for a frame with
    the two camera-following layers (shadow.x = 2), layer 1 from lightViewProjFar."""
    s, keep = _scene_struct(scene)
    keep = _drawn(s, keep, ndraw, draw_instances)
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    layers = int(lib().orc_shadow_layers(_p(frame)))
    out = np.zeros((layers, S, S) if layers > 1 else (S, S), np.float32)
    lib().orc_shadow_render(C.byref(s), _p(frame), S, _p(out))
    return out


def sun_tap(frame: np.ndarray, shadow: np.ndarray, x) -> float:
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    shadow = np.ascontiguousarray(shadow, dtype=np.float32)
    p = np.ascontiguousarray(x, dtype=np.float32)
    return float(lib().orc_sun_tap(_p(frame), _p(shadow), shadow.shape[-1], _p(p)))


def vox_sun(vox: dict, frame: np.ndarray, shadow: np.ndarray) -> None:
    """voxSun over a built world (vox from vox_build): fills vox['sunvis'] in place."""
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    shadow = np.ascontiguousarray(shadow, dtype=np.float32)
    vx = _vox_struct(vox)
    lib().orc_vox_sun(C.byref(vx), _p(frame), _p(shadow), shadow.shape[-1])


def bounce_dirs(rays: int) -> np.ndarray:
    """sfDir(i, rays) (bounce.ts:147-152) as the library tabulates it: the f32 steps of the shader, cos and sin of the
    f32 phi in double precision (the shader's are implementation-defined)."""
    f = np.float32
    libm = C.CDLL(C.util.find_library("m") or "libm.so.6")   # the C library's cos / sin, as the library's host code
    libm.cos.restype = libm.sin.restype = C.c_double
    libm.cos.argtypes = libm.sin.argtypes = [C.c_double]
    out = np.zeros((rays, 4), np.float32)
    for i in range(rays):
        fi, fn = f(i), f(rays)
        z = f(f(1.0) - (f(2.0) * fi + f(1.0)) / fn)
        zz = f(f(1.0) - z * z)
        r = f(np.sqrt(zz if zz > 0 else f(0.0)))
        xi = f(fi * f(0.618033988749))
        fr = f(xi - f(np.floor(xi)))
        phi = f(f(f(2.0) * f(3.14159265)) * fr)
        out[i] = (f(r * f(libm.cos(float(phi)))), f(r * f(libm.sin(float(phi)))), z, 0.0)
    return out


class Bounce:
    """The oracle's multi-bounce volume state (orc_bounce) across frames."""

    def __init__(self, vox: dict, cell: float = 1.2, dims=(32, 16, 32), rays: int = 16, div: int = 2,
                 objects: bool = False):
        """objects: the token obj (phase 31); the dynamic layer in vox['dyn'] at each frame receives the previous
        volume and is read by the volume's irradiance rays."""
        dx, dy, dz = dims
        self.dirs = bounce_dirs(rays)
        texels = dx * dy * (6 * dz + 1)
        self.vol = [np.zeros(texels * 4, np.float32), np.zeros(texels * 4, np.float32)]
        self.list = np.zeros(4 + dx * dy * dz, np.uint32)
        self.b = OrcBounce(np.float32(cell), np.float32(vox["v0"]), dx, dy, dz, rays, div, _p(self.dirs),
                           (C.c_void_p * 2)(_p(self.vol[0]), _p(self.vol[1])), _p(self.list), 1 if objects else 0)

    def frame(self, vox: dict, frame: np.ndarray) -> np.ndarray:
        """One frame over a built world; returns (and stores in vox['bn_inj']) the injected irradiance."""
        frame = np.ascontiguousarray(frame, dtype=np.float32)
        inj = np.zeros(vox["max_voxels"] * 6, np.float32)
        vx = _vox_struct(vox)
        vx.bn_inj = None
        lib().orc_bounce_frame(C.byref(self.b), C.byref(vx), _p(frame), _p(inj))
        vox["bn_inj"] = inj
        return inj


class WorldState:
    """What a world-probe solve keeps from one solve to the next (the hash tables, parents and the c0 history)."""

    def __init__(self, lay: dict):
        H0 = lay["casc"][0]["hash_mask"] + 1
        cap0 = lay["casc"][0]["cap"]
        self.keys = np.zeros(lay["hash_total"], np.uint32)
        self.slot_probe = np.zeros(lay["hash_total"], np.uint32)
        self.parents = np.zeros(lay["probes_total"] * 8, np.uint32)
        self.hist_tab = np.zeros(2 * H0, np.uint32)
        self.hist_grid = np.zeros(2 * cap0 * 4, np.int32)
        self.hist_sh = np.zeros(2 * cap0 * 32, np.float32)
        self.hist_par = 0


def wlayout_struct(lay: dict) -> OrcWLayout:
    wl = OrcWLayout()
    wl.base = layout_struct(lay)
    for i, c in enumerate(lay["casc"]):
        wl.hash_off[i], wl.hash_mask[i] = c["hash_off"], c["hash_mask"]
    wl.hash_total, wl.relocate = lay["hash_total"], lay["relocate"]
    return wl


def world_solve(vox: dict, lay: dict, state: WorldState, frame: np.ndarray, depth: np.ndarray, normal: np.ndarray,
                want_hit: bool = False, tag: np.ndarray = None) -> dict:
    """One world-probe solve (orc_world_solve) over a built voxel world; `state` carries over between solves.
    tag: the G-buffer's style tags (H x W bytes: 255 toon, 128 object, 0), or None (all photoreal)."""
    H, W = depth.shape
    wl = wlayout_struct(lay)
    cap0 = lay["casc"][0]["cap"]
    out = {"probes": np.zeros(lay["probes_total"], PROBE_DTYPE), "rad": np.zeros((lay["rays_total"], 4), np.float32),
           "sh": np.zeros((cap0, 32), np.float32), "irr": np.zeros((H, W, 4), np.float32),
           "counts": np.zeros(80, np.uint32)}
    if want_hit:
        out["hit"] = np.zeros((lay["rays_total"], 4), np.uint32)
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    normal = np.ascontiguousarray(normal, dtype=np.float32)
    tag = None if tag is None else np.ascontiguousarray(tag, dtype=np.uint8)
    g = OrcGbuf(_p(frame), W, H, _p(depth), _p(normal), None if tag is None else _p(tag))
    o = OrcRcOut(_p(out["probes"]), _p(out["rad"]), _p(out["sh"]), _p(out["irr"]), _p(out["counts"]),
                 _p(out["hit"]) if want_hit else None)
    ws = OrcWState(_p(state.keys), _p(state.slot_probe), _p(state.parents), _p(state.hist_tab), _p(state.hist_grid),
                   _p(state.hist_sh), state.hist_par)
    vx = _vox_struct(vox)
    lib().orc_world_solve(C.byref(vx), C.byref(wl), C.byref(g), C.byref(ws), C.byref(o))
    state.hist_par = ws.hist_par
    out["keys"] = state.keys.copy()
    out["slot_probe"] = state.slot_probe.copy()
    out["parents"] = state.parents.copy()
    return out


def hash32(x: int) -> int:
    return int(lib().orc_hash32(C.c_uint32(x)))


def lod_for(frame: np.ndarray, dist: float) -> int:
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    return int(lib().orc_lod_for(_p(frame), C.c_float(dist)))


class Dyn:
    """The dynamic layer (oracle/dyn.c, dynlayer.ts) of a voxel world built by vox_build: its arrays laid out as the
    CUDA path's (gi_dyn_read_state).  Set vox["dyn"] = this to make the cascades' traces read it."""

    def __init__(self, vox: dict, bricks: int = 512, albedo: bool = False):
        nptr = vox["levels"] * vox["G"] ** 3
        self.nb = bricks
        self.arrays = {"hdr": np.zeros(64, np.uint32), "ptr": np.zeros(nptr, np.uint32),
                       "bits": np.zeros(2 * nptr // 32, np.uint32), "meta": np.zeros(bricks, np.uint32),
                       "mask": np.zeros(bricks * 16, np.uint32), "data": np.zeros(bricks * 512 * 13, np.uint32)}
        a = self.arrays
        self.struct = OrcDyn(bricks, 1 if albedo else 0, _p(a["hdr"]), _p(a["ptr"]), _p(a["bits"]), _p(a["meta"]),
                             _p(a["mask"]), _p(a["data"]))
        vx = _vox_struct(vox)
        lib().orc_dyn_init(C.byref(vx), C.byref(self.struct))

    def build(self, scene, vox: dict, first: int, end: int, frame: np.ndarray, shadow: np.ndarray = None) -> None:
        """One build of the dynamic triangles [first, end) in the windows of `vox` (its origins)."""
        s, keep = _scene_struct(scene)
        frame = np.ascontiguousarray(frame, dtype=np.float32)
        vx = _vox_struct({**vox, "dyn": None})
        sm = None if shadow is None else np.ascontiguousarray(shadow, dtype=np.float32)
        lib().orc_dyn_build(C.byref(s), C.byref(vx), C.byref(self.struct), first, end, _p(frame),
                            _p(sm) if sm is not None else None, 0 if sm is None else sm.shape[-1])

    def trace(self, vox: dict, o, d, t0: float, t1: float, k: float) -> np.ndarray:
        """traceDyn of one segment: covered radiance rgb and coverage."""
        vx = _vox_struct({**vox, "dyn": self})
        oo, dd = np.asarray(o, np.float32).copy(), np.asarray(d, np.float32).copy()
        out = np.zeros(4, np.float32)
        lib().orc_trace_dyn(C.byref(vx), _p(oo), _p(dd), t0, t1, k, _p(out))
        return out


def log2(x: float) -> float:
    return float(lib().orc_log2(x))
