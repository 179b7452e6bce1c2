"""The sun shadow map drawn on the GPU against the oracle's brute-force raster, bit for bit, on triangles chosen to
stress the raster's tile skipping: slivers, near-degenerate and huge triangles, vertices far outside the map."""
import numpy as np
import pytest

from oracle import bind
from rtgi import frame as fr, gpu, scenes

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
