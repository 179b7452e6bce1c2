"""Parity of the world work items (gi_vox_set_world / gi_vox_set_items; world.ts, voxel.ts:270-288) with the oracle:
a room placed at four instances, its chunks voxelised from their finest window, the clustered copies at the coarse
levels.  The voxel state and a whole solve are compared bit for bit; a world of one instance must equal the plain
build; stale graphs and bad items are refused."""
import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, configs, frame as fr, gpu, scenes, world as W

pytestmark = pytest.mark.gpu

ROOM_V = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}
INSTANCES = [(0, 0, 0), (12, 0, 0), (-14, 0, 3), (0, 0, 26)]
STATE = ("hdr", "ptr", "occ", "base", "code", "attr", "plane")


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.destroy()


def _gpu_world(ctx, s, s2, w, v, p, W_, H_, F):
    sg = gpu.SceneGpu(ctx, s2)
    sg.set_draw_count(s.triangle_count)   # the clustered copies are voxelised, not drawn
    vw = gpu.VoxWorld(sg, v)
    vw.set_world(w)
    rc = gpu.Rc(ctx, p, W_, H_)
    try:
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        vw.update(s.camera.eye)
        rc.solve(vw)
        out = {"state": vw.read_state(), "irr": rc.read_irradiance(),
               "depth": rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H_, W_),
               "normal": rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H_, W_, 4).astype(np.float32)}
        return out, (sg, vw, rc)
    except Exception:
        for h in (rc, vw, sg):
            h.destroy()
        raise


def test_world_items_parity(ctx):
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    p = configs.parse_config("screen-8-voxel-f32-dda256", {"cascades": 4})
    s2, w = W.with_world(s, INSTANCES, float(v.v0), v.levels)
    W_, H_ = 240, 160
    F = gi_cases._frame(s, W_, H_, p, sun_e=fr.SUN_E, sky=fr.SKY)
    g, handles = _gpu_world(ctx, s, s2, w, v, p, W_, H_, F)
    try:
        st = bind.vox_build(s2, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye, world=w)
        for k in STATE:
            assert np.array_equal(g["state"][k], st[k]), f"voxel {k} differs from the oracle"
        assert st["hdr"][9] > 0 and st["hdr"][10] > 0
        depth, normal, _ = bind.raster_gbuffer(s, F, W_, H_)   # the static scene, as drawn
        assert np.array_equal(g["depth"].view(np.uint32), depth.view(np.uint32))
        out = bind.rc_solve(st, configs.cascade_layout(p, W_, H_), F, g["depth"], g["normal"])
        assert np.array_equal(g["irr"].view(np.uint32), out["irr"].view(np.uint32)), "irradiance differs"
        assert g["irr"][..., :3].max() > 0
    finally:
        for h in reversed(handles):
            h.destroy()


def test_single_instance_world_equals_plain_build(ctx):
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    s1, w1 = W.with_world(s, [(0, 0, 0)], float(v.v0), v.levels)
    sg0, sg1 = gpu.SceneGpu(ctx, s), gpu.SceneGpu(ctx, s1)   # s1 = s + the clustered rows (unused by instance 0)
    v0, v1 = gpu.VoxWorld(sg0, v), gpu.VoxWorld(sg1, v)
    try:
        v0.update(s.camera.eye)
        v0.encode()
        plain = v0.read_state()
        v1.set_world(w1)
        v1.update(s.camera.eye)
        v1.encode()
        world = v1.read_state()
        for k in STATE:
            assert np.array_equal(plain[k], world[k]), k
    finally:
        for h in (v0, v1, sg0, sg1):
            h.destroy()


def test_items_are_checked_and_stale_graphs_refused(ctx):
    import torch
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    p = configs.parse_config("screen-8-voxel-f32-dda64", {"cascades": 2})
    s2, w = W.with_world(s, INSTANCES, float(v.v0), v.levels)
    sg = gpu.SceneGpu(ctx, s2)
    sg.set_draw_count(s.triangle_count)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, 64, 48)
    try:
        vw.set_world(w)
        bad = [np.array([[0, 0x80000000, 9, 0]], np.uint32),          # no instance 9
               np.array([[0, 0x80000000, 0, 7]], np.uint32),          # no level 7
               np.array([[1, 0x80000000, 0, 0]], np.uint32)]          # does not start at thread 0
        for rec in bad:
            with pytest.raises(_lib.GiError):
                _lib.call("gi_vox_set_items", vw.handle, rec.ctypes.data, 1, 4)
        with pytest.raises(_lib.GiError):   # a range past the rows
            rec = np.array([[0, 0x80000000 | (w.rows - 2), 0, 0]], np.uint32)
            _lib.call("gi_vox_set_items", vw.handle, rec.ctypes.data, 1, 4)
        F = gi_cases._frame(s, 64, 48, p)
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        vw.update(s.camera.eye)
        stream = torch.cuda.Stream()
        rc.graph_capture(vw, stream)
        rc.graph_launch(stream)
        stream.synchronize()
        vw.update(s.camera.eye)   # new items (the same ones): the graph holds the old ones
        with pytest.raises(_lib.GiError):
            rc.graph_launch(stream)
        rc.graph_capture(vw, stream)
        rc.graph_launch(stream)
        stream.synchronize()
    finally:
        for h in (rc, vw, sg):
            h.destroy()


def test_instanced_rasters(ctx):
    """The rasters draw the static rows at every instance (gi_scene_set_draw_instances): the G-buffer and the sun's
    shadow map of four room instances seen from above, bit-exact with the oracle's rasters."""
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    s2, w = W.with_world(s, INSTANCES, float(v.v0), v.levels)
    cam = fr.Camera((-18.0, 22.0, -16.0), (6.0, 0.0, 12.0), 60, 0.05)
    W_, H_ = 200, 150
    p = configs.parse_config("screen-8-voxel-f32-dda64", {"cascades": 2})
    bmin = np.min([np.asarray(s.positions).min(0) + o for o in INSTANCES], axis=0)
    bmax = np.max([np.asarray(s.positions).max(0) + o for o in INSTANCES], axis=0)
    F = fr.pack_frame(fr.FrameParams(cam=cam, width=W_, height=H_, sun_dir=(0.3, 1.0, 0.2), cascades=p.cascades, P=p.P,
                                     light_view_proj=fr.scene_sun_view_proj(tuple(map(float, bmin)), tuple(map(float, bmax)),
                                                                            (0.3, 1.0, 0.2)),
                                     shadow_bias=fr.SHADOW_BIAS))
    sg = gpu.SceneGpu(ctx, s2)
    rc = gpu.Rc(ctx, p, W_, H_)
    try:
        sg.set_draw_count(s.triangle_count)
        sg.set_draw_instances(INSTANCES)
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        rc.render_shadow(sg, 256)
        depth = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H_, W_)
        normal = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H_, W_, 4).astype(np.float32)
        shadow = rc.read_shadow()
        d0, n0, tri = bind.raster_gbuffer(s2, F, W_, H_, ndraw=s.triangle_count, draw_instances=INSTANCES)
        assert np.array_equal(depth.view(np.uint32), d0.view(np.uint32))
        assert np.array_equal(normal.astype(np.float16).view(np.uint16), n0.astype(np.float16).view(np.uint16))
        sm = bind.shadow_render(s2, F, 256, ndraw=s.triangle_count, draw_instances=INSTANCES)
        assert np.array_equal(shadow.view(np.uint32), sm.view(np.uint32))
        inst_of = tri[tri != 0xFFFFFFFF] // s.triangle_count
        assert len(set(inst_of.tolist())) >= 3            # several instances are in view
        sg.set_draw_instances(None)                       # back to one draw
        rc.render_gbuffer(sg)
        d1 = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H_, W_)
        assert (d1 > 0).sum() < (depth > 0).sum()
    finally:
        rc.destroy()
        sg.destroy()
