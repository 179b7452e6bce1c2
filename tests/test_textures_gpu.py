"""Base colour textures on the GPU (gi_scene_set_textures) against the oracle: the room with striped boxes and
alpha-masked lattice panels — the voxel state (the alpha test cutting the panels' holes, the sampled albedo), the
G-buffer and shadow map, and the whole solve's irradiance, bit for bit."""
import dataclasses

import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, configs, frame as fr, gpu, scenes

pytestmark = pytest.mark.gpu

VOX = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}
STATE = ("hdr", "ptr", "occ", "base", "code", "attr", "plane", "sunvis")


def _run(s, W=256, H=192, shadow=512):
    p = configs.parse_config("screen-8-voxel-f32-dda256", {"cascades": 4})
    v = configs.vox_params(VOX)
    F = gi_cases._frame(s, W, H, p, sun_e=fr.SUN_E, sky=fr.SKY, shadow=True)
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    try:
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        rc.render_shadow(sg, shadow)
        vw.update(s.camera.eye)
        rc.solve(vw)
        g = {"vox": vw.read_state(), "irr": rc.read_irradiance(), "shadow": rc.read_shadow(),
             "depth": rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H, W),
             "normal": rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H, W, 4).astype(np.float32)}
    finally:
        for h in (rc, vw, sg, ctx):
            h.destroy()
    return g, p, v, F


def test_textured_scene_parity():
    s = scenes.textured_scene()
    g, p, v, F = _run(s)
    depth, normal, _ = bind.raster_gbuffer(s, F, 256, 192)
    assert np.array_equal(g["depth"].view(np.uint32), depth.view(np.uint32)), "G-buffer depth"
    assert np.array_equal(g["normal"], normal), "G-buffer normal"
    shadow = bind.shadow_render(s, F, 512)
    assert np.array_equal(g["shadow"].view(np.uint32), shadow.view(np.uint32)), "shadow map"
    st = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye)
    bind.vox_sun(st, F, shadow)
    nb, nv = int(st["hdr"][0]), int(st["hdr"][1])
    for k in STATE:
        n = {"occ": nb * 16, "base": nb, "code": nb, "attr": nv * 4, "plane": nv, "sunvis": nv}.get(k)
        a, b = g["vox"][k], st[k]
        if n is not None:
            a, b = a[:n], b[:n]
        assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32)), f"voxel {k}"
    o = bind.rc_solve(st, configs.cascade_layout(p, 256, 192), F, depth, normal)
    assert np.array_equal(g["irr"].view(np.uint32), o["irr"].view(np.uint32)), "irradiance"
    # the textures matter: without them the panels are solid and the boxes take their factor
    g0, *_ = _run(dataclasses.replace(s, textures=None, uvs=None))
    assert int(g0["vox"]["hdr"][1]) > nv
    assert not np.array_equal(g0["irr"], g["irr"])


def test_graph_refused_after_the_textures_change():
    """A captured solve holds the scene's buffers: replacing the textures (or a draw count) afterwards makes the replay
    refuse until the solve is captured again."""
    s = scenes.textured_scene(16)
    p = configs.parse_config("screen-8-voxel-f32", {"cascades": 2})
    v = configs.vox_params(VOX)
    F = gi_cases._frame(s, 64, 48, p, sun_e=fr.SUN_E, sky=fr.SKY)
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, 64, 48)
    import torch
    st = torch.cuda.Stream()
    try:
        rc.set_frame(F, st)
        rc.render_gbuffer(sg, st)
        vw.update(s.camera.eye)
        rc.graph_capture(vw, st)
        rc.graph_launch(st)
        sg.set_textures(s.textures[::-1].copy(), s.uvs)
        with pytest.raises(_lib.GiError) as e:
            rc.graph_launch(st)
        assert e.value.status == _lib.GI_ERR_STATE
        rc.graph_capture(vw, st)
        rc.graph_launch(st)
        sg.set_draw_count(s.triangle_count - 2)
        with pytest.raises(_lib.GiError):
            rc.graph_launch(st)
        st.synchronize()
    finally:
        for h in (rc, vw, sg, ctx):
            h.destroy()
