"""ctypes binding of libgi_b200.so (include/gi.h).  There is no fallback: if the library is missing or the device is
not a B200 the calls raise, so nothing runs a CPU path in its place."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libgi_b200.so")

GI_OK, GI_ERR_INVALID, GI_ERR_OOM, GI_ERR_CUDA, GI_ERR_TIMEOUT, GI_ERR_OVERFLOW, GI_ERR_STATE = 0, -1, -2, -3, -4, -5, -6
GI_ATLAS_F32, GI_ATLAS_F16, GI_ATLAS_BF16 = 0, 1, 2
(GI_RC_PROBES, GI_RC_RAD, GI_RC_SH, GI_RC_DEPTH, GI_RC_NORMAL, GI_RC_HITS, GI_RC_RAD_TRACED, GI_RC_SHADOW, GI_RC_BOUNCE_VOL,
 GI_RC_BOUNCE_INJ, GI_RC_BOUNCE_LIST, GI_RC_WORLD_KEYS, GI_RC_WORLD_SLOTS, GI_RC_WORLD_PARENTS, GI_RC_WORLD_STATE,
 GI_RC_TAG) = range(16)
GI_RELOCATE_GBUFFER, GI_RELOCATE_NONE, GI_RELOCATE_VOXEL = 0, 1, 2

# Every symbol include/gi.h declares, with its ctypes signature (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "gi_version": (C.c_int, []),
    "gi_status_string": (C.c_char_p, [C.c_int]),
    "gi_last_error": (C.c_char_p, []),
    "gi_ctx_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "gi_ctx_destroy": (C.c_int, [_P]),
    "gi_scene_upload": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32, C.POINTER(_P)]),
    "gi_scene_update_vertices": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "gi_scene_set_textures": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, _P]),
    "gi_scene_destroy": (C.c_int, [_P]),
    "gi_vox_create": (C.c_int, [_P, _P, C.POINTER(_P)]),
    "gi_vox_update": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "gi_vox_build": (C.c_int, [_P, _P]),
    "gi_vox_read_counters": (C.c_int, [_P, _P, _P]),
    "gi_vox_debug_hold_scan": (C.c_int, [_P, C.c_int32]),
    "gi_vox_used_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "gi_vox_read_state": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "gi_vox_destroy": (C.c_int, [_P]),
    "gi_vox_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "gi_scene_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "gi_vox_build_noalloc": (C.c_int, [_P, C.POINTER(C.c_double), _P, _P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32,
                                       _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "gi_rc_create": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    "gi_vox_set_world": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32]),
    "gi_vox_set_items": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32]),
    "gi_scene_set_draw_count": (C.c_int, [_P, C.c_uint32]),
    "gi_scene_set_draw_instances": (C.c_int, [_P, _P, C.c_uint32]),
    "gi_rc_create_world": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    "gi_rc_set_frame": (C.c_int, [_P, _P, _P]),
    "gi_rc_set_gbuffer": (C.c_int, [_P, _P, _P, _P]),
    "gi_rc_set_gbuffer_f16": (C.c_int, [_P, _P, _P, _P]),
    "gi_rc_set_gbuffer_rgb16f": (C.c_int, [_P, _P, _P, _P]),
    "gi_rc_set_gbuffer_tag": (C.c_int, [_P, _P, _P]),
    "gi_rc_render_gbuffer": (C.c_int, [_P, _P, _P]),
    "gi_rc_render_shadow": (C.c_int, [_P, _P, C.c_uint32, _P]),
    "gi_rc_set_bounce": (C.c_int, [_P, _P, _P]),
    "gi_vox_build_sun": (C.c_int, [_P, _P, _P]),
    "gi_rc_solve": (C.c_int, [_P, _P, _P]),
    "gi_solve": (C.c_int, [_P, _P, _P]),
    "gi_rc_read_irradiance": (C.c_int, [_P, _P, _P]),
    "gi_rc_read_irradiance_raw": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "gi_rc_read_irradiance_async": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "gi_rc_read_counts": (C.c_int, [_P, _P, _P]),
    "gi_rc_set_stats": (C.c_int, [_P, C.c_uint32]),
    "gi_rc_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "gi_rc_read_buffer": (C.c_int, [_P, C.c_int, _P, C.c_size_t, _P]),
    "gi_rc_buffer_bytes": (C.c_int, [_P, C.c_int, C.POINTER(C.c_size_t)]),
    "gi_rc_set_debug_hits": (C.c_int, [_P, C.c_int]),
    "gi_rc_merge_gather_f64": (C.c_int, [_P, _P]),
    "gi_rc_merge_gather_f64_rounded": (C.c_int, [_P, C.c_uint32, _P]),
    "gi_scene_set_raster_capacity": (C.c_int, [_P, C.c_uint32]),
    "gi_scene_rigid_define": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32]),
    "gi_scene_rigid_upload": (C.c_int, [_P, _P, _P]),
    "gi_scene_rigid_apply": (C.c_int, [_P, _P]),
    "gi_rc_graph_capture_frame": (C.c_int, [_P, _P, _P, _P, _P]),
    "gi_rc_set_tuning": (C.c_int, [_P, _P]),
    "gi_rc_get_tuning": (C.c_int, [_P, _P]),
    "gi_vox_set_tuning": (C.c_int, [_P, _P]),
    "gi_vox_get_tuning": (C.c_int, [_P, _P]),
    "gi_rc_read_irradiance_f64": (C.c_int, [_P, _P, _P]),
    "gi_rc_graph_capture": (C.c_int, [_P, _P, _P]),
    "gi_rc_graph_launch": (C.c_int, [_P, _P]),
    "gi_batch_create": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(_P)]),
    "gi_batch_capture": (C.c_int, [_P, _P]),
    "gi_batch_capture_passes": (C.c_int, [_P, _P]),
    "gi_batch_launch": (C.c_int, [_P, _P]),
    "gi_batch_destroy": (C.c_int, [_P]),
    "gi_rc_set_timing": (C.c_int, [_P, C.c_int]),
    "gi_rc_pass_times": (C.c_int, [_P, _P]),
    "gi_rc_destroy": (C.c_int, [_P]),
    "gi_scene_set_static_count": (C.c_int, [_P, C.c_uint32]),
    "gi_dyn_create": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    "gi_dyn_build": (C.c_int, [_P, _P, _P]),
    "gi_dyn_read_counters": (C.c_int, [_P, _P, _P]),
    "gi_dyn_read_state": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "gi_dyn_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "gi_dyn_destroy": (C.c_int, [_P]),
    "gi_rc_set_dyn": (C.c_int, [_P, _P]),
    "gi_rc_set_objects": (C.c_int, [_P, C.c_int]),
}


class GiError(RuntimeError):
    """A non-zero gi_status (the reference throws `new Error(msg)` at the same places)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} [{status}]")
        self.status = status


class GiVoxParams(C.Structure):
    _fields_ = [("v0", C.c_double), ("levels", C.c_uint32), ("G", C.c_uint32), ("max_bricks", C.c_uint32),
                ("max_voxels", C.c_uint32), ("dyn_bricks", C.c_uint32), ("reserved", C.c_uint32)]


class GiRcParams(C.Structure):
    _fields_ = [("cascades", C.c_uint32), ("P", C.c_uint32), ("k_interval", C.c_float), ("vox_scale", C.c_float),
                ("vox_offset", C.c_float), ("vox_skip", C.c_float), ("level_map", C.c_float), ("res_cap", C.c_uint32),
                ("dda_cap", C.c_uint32), ("stats", C.c_uint32), ("atlas", C.c_uint32), ("f32_out", C.c_uint32),
                ("irr_f16", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class GiRcTuning(C.Structure):
    _fields_ = [("trace_order", C.c_uint32), ("trace_rays", C.c_uint32), ("trace_blocks", C.c_uint32),
                ("gather_shape", C.c_uint32), ("merge_threads", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class GiVoxTuning(C.Structure):
    _fields_ = [("chunk_cells", C.c_uint32), ("blocks", C.c_uint32), ("reserved", C.c_uint32 * 6)]


class GiWorldParams(C.Structure):
    _fields_ = [("relocate", C.c_uint32), ("caps", C.c_uint32 * 8), ("reserved", C.c_uint32 * 3)]


class GiBounceParams(C.Structure):
    _fields_ = [("cell", C.c_float), ("dx", C.c_uint32), ("dy", C.c_uint32), ("dz", C.c_uint32), ("rays", C.c_uint32),
                ("div", C.c_uint32), ("reserved", C.c_uint32 * 2)]


_lib = None


def build(force: bool = False) -> str:
    """Compiles the library with nvcc (real-time-gi-lab_b200/build.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("gi_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def load(path: str = LIB_PATH):
    """Loads the library; builds it first only when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if path == LIB_PATH and os.path.exists(os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")):
        build()   # only when missing or older than its sources (build.py checks)
    if not os.path.exists(path):
        raise ImportError(f"libgi_b200.so not found at {path}; build it with real-time-gi-lab_b200/build.py")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "") -> None:
    if status != GI_OK:
        msg = load().gi_last_error().decode(errors="replace")
        raise GiError(status, msg or what or load().gi_status_string(status).decode())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)
