"""Host logic of the precision study and the moving boxes, on the CPU."""
import numpy as np
import torch

from rtgi import movers, precision, scenes, serve


def _small_base():
    b = scenes.Builder([scenes.Material("ground", (0.5, 0.5, 0.5, 1.0))])
    b.quad([-5, 0, 5], [5, 0, 5], [5, 0, -5], [-5, 0, -5])
    return b.scene("ground", scenes.Camera((0, 1.7, 0), (5, 1.5, 0), 60, 0.05))


def test_moving_boxes_are_rigid_and_wrap():
    base = _small_base()
    s, objs = movers.with_moving_boxes(base, 5, scenes.PCG32(3, stream=41), area=(2.0, -1.0, 3.0, 2.0))
    assert s.triangle_count == base.triangle_count + 5 * 12
    assert objs.first == base.positions.shape[0]
    p0, n0 = objs.pose(0.0)
    np.testing.assert_allclose(p0, s.positions[objs.first:], atol=1e-6)
    p1, n1 = objs.pose(7.3)
    a, b = p0.reshape(5, -1, 3).astype(np.float64), p1.reshape(5, -1, 3).astype(np.float64)
    da = np.linalg.norm(a[:, :, None] - a[:, None], axis=-1)
    db = np.linalg.norm(b[:, :, None] - b[:, None], axis=-1)
    np.testing.assert_allclose(da, db, atol=1e-4)                     # rigid
    np.testing.assert_allclose(np.linalg.norm(n1, axis=-1), 1.0, atol=1e-6)
    c = b.mean(axis=1)
    ax, az, hx, hz = objs.area
    assert (np.abs(c[:, 0] - ax) <= hx + 1.0).all() and (np.abs(c[:, 2] - az) <= hz + 1.0).all()
    np.testing.assert_allclose(c[:, 1], a.mean(axis=1)[:, 1], atol=1e-5)   # no vertical motion


def test_serving_scene_unchanged_by_the_movers_module():
    spec = scenes.batch_spec(2)
    s1, o1 = serve.serving_scene(spec, 9)
    s2, o2 = serve.serving_scene(spec, 9)
    assert np.array_equal(s1.positions, s2.positions) and o1.first == o2.first
    assert o1.area == (0.0, 0.0, 20.0, 20.0)


def test_error_stats_quantiles_and_norms():
    st = precision.ErrorStats(torch, torch.device("cpu"))
    ref = torch.ones((4, 8, 4), dtype=torch.float64)
    ref[0, 0, 3] = 0.0                       # background pixel: not counted
    x = (ref * (1 + 1e-3)).to(torch.float32)
    x[..., 3] = ref[..., 3].to(torch.float32)
    st.add(x, ref)
    s = st.summary()
    assert s["values"] == 31 * 3 and s["alpha_mismatch"] == 0
    assert 0.9e-3 < s["mean_rel"] < 1.1e-3 and 0.9e-3 < s["rel_l2"] < 1.1e-3
    assert 1e-3 <= s["p50_rel"] <= 10 ** -2.8 and 1e-3 <= s["p99_rel"] <= 10 ** -2.8
    x2 = x.clone()
    x2[1, 1, 3] = 0.0
    st.add(x2, ref)
    assert st.summary()["alpha_mismatch"] == 1


def test_colonnade_precision_scene():
    s, objs = precision.precision_scene(0, 64)
    assert s.triangle_count == scenes.colonnade_scene(0).triangle_count + 64 * 12
    p, v = precision.colonnade_params("f16")
    assert p.atlas == "f16" and p.cascades == 5 and v.levels == 4 and v.G == 16


def test_rigid_transforms_reproduce_pose():
    base = _small_base()
    s, objs = movers.with_moving_boxes(base, 6, scenes.PCG32(5, stream=41))
    rest_p = s.positions[objs.first:].astype(np.float64).reshape(6, -1, 3)
    rest_n = s.normals[objs.first:].astype(np.float64).reshape(6, -1, 3)
    for t in (0.0, 0.4, 13.0):
        m = objs.transforms(t).astype(np.float64).reshape(6, 3, 4)
        p = np.einsum("oij,ovj->ovi", m[:, :, :3], rest_p) + m[:, None, :, 3]
        n = np.einsum("oij,ovj->ovi", m[:, :, :3], rest_n)
        pp, nn = objs.pose(t)
        np.testing.assert_allclose(p.reshape(-1, 3), pp, atol=2e-5)
        np.testing.assert_allclose(n.reshape(-1, 3), nn, atol=1e-6)


def test_f64_storage_rounding_in_the_oracle():
    """The oracle's FP64 merge with the atlas storage of some cascades rounded to f16.  Cascade 0 alone rounds only its
    traced intervals (its merged radiances feed projectSH unstored), so it equals rounding them beforehand with numpy's
    float16 (round to nearest even).  Every cascade rounded moves the irradiance by about f16's relative step."""
    from oracle import bind
    from rtgi import configs, frame as fr
    s = scenes.room_scene(0)
    W, H = 96, 64
    v = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    st = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye)
    q = configs.parse_config("screen-8-voxel-f32", {"cascades": 3})
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=fr.SUN_E, sky=fr.SKY,
                                     cascades=q.cascades, P=q.P))
    depth, normal, _ = bind.raster_gbuffer(s, F, W, H)
    nrm = normal.astype(np.float16).astype(np.float32)
    lay = configs.cascade_layout(q, W, H)
    o = bind.rc_solve(st, lay, F, depth, nrm, merge=False)
    args = (lay, F, depth, nrm, o["probes"])
    exact = bind.merge_gather_f64(*args, o["rad_traced"])
    c0 = lay["casc"][0]
    a, n = c0["rad_off"], c0["tiles_x"] * c0["tiles_y"] * c0["res"] ** 2
    pre = o["rad_traced"].copy()
    pre[a:a + n] = pre[a:a + n].astype(np.float16).astype(np.float32)
    assert np.array_equal(bind.merge_gather_f64(*args, o["rad_traced"], f16_cascades=1), bind.merge_gather_f64(*args, pre))
    every = bind.merge_gather_f64(*args, o["rad_traced"], f16_cascades=0b111)
    valid = exact[..., 3] > 0
    assert valid.any() and np.array_equal(every[..., 3], exact[..., 3])
    d, r = (every - exact)[..., :3][valid], exact[..., :3][valid]
    rel_l2 = np.sqrt((d * d).sum() / (r * r).sum())
    assert 1e-6 < rel_l2 < 2.0 ** -10
