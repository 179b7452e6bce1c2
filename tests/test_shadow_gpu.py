"""The sun shadow map drawn on the GPU against the oracle's brute-force raster, bit for bit, on triangles chosen to
stress the raster's tile skipping: slivers, near-degenerate and huge triangles, vertices far outside the map."""
import numpy as np
import pytest

from oracle import bind
from rtgi import _lib, frame as fr, gpu, scenes

pytestmark = pytest.mark.gpu


def _stress_scene(seed=4, n=3000):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-10, 10, (n, 3))
    kind = rng.integers(0, 4, n)
    b = a + rng.uniform(-3, 3, (n, 3))
    c = a + rng.uniform(-3, 3, (n, 3))
    c[kind == 1] = a[kind == 1] + (b[kind == 1] - a[kind == 1]) * rng.uniform(0, 1, (np.sum(kind == 1), 1)) \
        + rng.normal(0, 1e-4, (np.sum(kind == 1), 3))                       # slivers
    b[kind == 2] = a[kind == 2] + rng.uniform(-60, 60, (np.sum(kind == 2), 3))   # huge, partly off the map
    c[kind == 3] = a[kind == 3] + 1e-6                                       # near-degenerate
    pos = np.stack([a, b, c], 1).reshape(-1, 3).astype(np.float32)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (pos.shape[0], 1))
    tri = np.zeros((n, 4), np.uint32)
    tri[:, :3] = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    mats = [scenes.Material("grey", (0.5, 0.5, 0.5, 1.0))]
    return scenes.Scene("shadow-stress", pos, nrm, tri, mats, scenes.Camera((0, 5, 20), (0, 0, 0), 60, 0.05),
                        sun_dir=(-0.4, 1.0, 0.3))


@pytest.mark.parametrize("size", [256, 1024])
def test_shadow_map_stress(size):
    s = _stress_scene()
    bmin, bmax = [-12.0, -12.0, -12.0], [12.0, 12.0, 12.0]   # the huge triangles reach past the light's window
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=64, height=64, sun_dir=s.sun_dir,
                                     light_view_proj=fr.scene_sun_view_proj(bmin, bmax, s.sun_dir),
                                     shadow_bias=fr.SHADOW_BIAS, cascades=2))
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s)
    rc = gpu.Rc(ctx, gpu_params(), 64, 64)
    try:
        rc.set_frame(F)
        rc.render_shadow(sg, size)
        got = rc.read_shadow()
    finally:
        for h in (rc, sg, ctx):
            h.destroy()
    ref = bind.shadow_render(s, F, size)
    assert (ref < 1.0).mean() > 0.2
    bad = got.view(np.uint32) != ref.view(np.uint32)
    assert not bad.any(), f"{bad.sum()} texels differ, first at {np.argwhere(bad)[:4].tolist()}"


def gpu_params():
    from rtgi import configs
    return configs.parse_config("screen-8-voxel-f32", {"cascades": 2})


def test_camera_following_layers_on_a_world():
    """An instanced world (the room at 121 instances 12 m apart, 130 m across) with the two camera-following layers
    (lighting.ts:93-126): both layers of the map, the voxels' sun visibility and the irradiance bit for bit with the
    oracle; some voxels lie outside layer 0 and read layer 1."""
    from rtgi import configs, world as W
    import gi_cases
    room = scenes.room_scene(0)
    inst = [(12.0 * i, 0.0, 12.0 * j) for j in range(-5, 6) for i in range(-5, 6)]
    inst.remove((0.0, 0.0, 0.0))
    inst.insert(0, (0.0, 0.0, 0.0))
    v = configs.vox_params({"v0": 0.16, "levels": 4, "G": 16, "maxBricks": 16384, "maxVoxels": 1 << 21})
    s2, w = W.with_world(room, inst, float(v.v0), v.levels)
    p = configs.parse_config("screen-8-voxel-f32-dda256", {"cascades": 3})
    Wd, Hd, S = 160, 120, 512
    eye = room.camera.eye
    near, far = fr.world_sun_view_projs(room.sun_dir, eye, S)
    F = gi_cases._frame(room, Wd, Hd, p, sun_e=fr.SUN_E, sky=fr.SKY)
    F = F.copy()
    F[64:80], F[140:156] = near, far
    F[156:160] = [2, fr.SHADOW_WORLD_BIAS[0], fr.SHADOW_WORLD_BIAS[1], 0]
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s2)
    sg.set_draw_count(room.triangle_count)
    sg.set_draw_instances(inst)
    vw = gpu.VoxWorld(sg, v)
    vw.set_world(w)
    rc = gpu.Rc(ctx, p, Wd, Hd)
    try:
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        rc.render_shadow(sg, S)
        vw.update(eye)
        rc.solve(vw)
        got_map, g_state, g_irr = rc.read_shadow(), vw.read_state(), rc.read_irradiance()
        depth = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(Hd, Wd)
        normal = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(Hd, Wd, 4).astype(np.float32)
    finally:
        for h in (rc, vw, sg, ctx):
            h.destroy()
    ref = bind.shadow_render(room, F, S, draw_instances=inst)
    assert got_map.shape == (2, S, S)
    assert (ref[1] < 1.0).any() and (ref[0] < 1.0).any()
    bad = got_map.view(np.uint32) != ref.view(np.uint32)
    assert not bad.any(), f"{bad.sum()} texels differ, first at {np.argwhere(bad)[:4].tolist()}"
    st = bind.vox_build(s2, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, eye, world=w)
    bind.vox_sun(st, F, ref)
    nv = int(min(st["hdr"][1], v.maxVoxels))
    assert np.array_equal(g_state["sunvis"][:nv].view(np.uint32), st["sunvis"][:nv].view(np.uint32)), "sun visibility"
    # some voxels are placed outside layer 0 (the coarse levels reach 164 m from the camera)
    M0 = np.array(near, np.float64).reshape(4, 4).T
    org = st["origin"]
    outside = 0
    for b in range(int(min(st["hdr"][0], v.maxBricks))):
        code = int(st["code"][b])
        L, bx, bz = code >> 27, (code >> 18) & 511, code & 511
        vs = v.v0 * 2 ** L
        x = (org[L, 0] * 8 + bx * 8 + 4) * vs
        z = (org[L, 2] * 8 + bz * 8 + 4) * vs
        q = M0 @ np.array([x, 0.0, z, 1.0])
        outside += abs(q[0]) > 1.0 or abs(q[1]) > 1.0
    assert outside > 0
    out = bind.rc_solve(st, configs.cascade_layout(p, Wd, Hd), F, depth, normal)
    assert np.array_equal(g_irr.view(np.uint32), out["irr"].view(np.uint32)), "irradiance differs"


def test_a_frame_asking_for_more_layers_than_the_map_is_refused():
    """A map drawn for one layer and a frame that asks for two: the solve is refused before any kernel reads past
    the map."""
    from rtgi import configs
    import gi_cases
    room = scenes.room_scene(0)
    p = configs.parse_config("screen-8-voxel-f32", {"cascades": 2})
    v = configs.vox_params({"v0": 0.16, "levels": 1, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 18})
    F = gi_cases._frame(room, 64, 48, p, sun_e=fr.SUN_E, sky=fr.SKY, shadow=True)
    ctx = gpu.Context(0)
    sg, rc = gpu.SceneGpu(ctx, room), gpu.Rc(ctx, p, 64, 48)
    vw = gpu.VoxWorld(sg, v)
    try:
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        rc.render_shadow(sg, 128)
        vw.update(room.camera.eye)
        rc.solve(vw)
        F2 = F.copy()
        F2[140:156] = F[64:80]
        F2[156] = 2
        rc.set_frame(F2)
        with pytest.raises(_lib.GiError) as e:
            rc.solve(vw)
        assert e.value.status == _lib.GI_ERR_STATE
        rc.render_shadow(sg, 128)      # drawn again for two layers: accepted
        rc.solve(vw)
    finally:
        for h in (rc, vw, sg, ctx):
            h.destroy()
