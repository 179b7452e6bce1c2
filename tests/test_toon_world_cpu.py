"""The world gather's receiving operator for toon pixels (rc.ts:877-926, style.ts:30-42) in the oracle: the G-buffer's
style tag selects it, the L0/L1 SH of the pixel's probes are interpolated with the irradiance's weights and put
through toonReceive; output alpha 2 + band + 2 contrast for toon pixels, 2 for other tagged ones, 1 photoreal; only
photoreal pixels count as black."""
import dataclasses

import numpy as np

from oracle import bind
from rtgi import configs, frame as fr, scenes

VOX = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}
W, H = 96, 64


def _solve(tag, style=(1.0, 1.0, 0.0)):
    s = scenes.room_scene(0)
    p = configs.parse_config("world-24-voxel-rc2-f32", {"cascades": 3, "caps": [4096, 2048, 1024] + [256] * 5})
    lay = configs.world_layout(p)
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=fr.SUN_E, sky=fr.SKY,
                                     cascades=p.cascades, P=p.P, s_min=p.sMin, lift=p.lift, style=style))
    depth, normal, tri = bind.raster_gbuffer(s, F, W, H)
    normal = normal.astype(np.float16).astype(np.float32)
    v = configs.vox_params(VOX)
    st = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye)
    return bind.world_solve(st, lay, bind.WorldState(lay), F, depth, normal, tag=tag), depth


def _recv(c0, c1y, c1z, c1x, n, soft):
    """toonReceive restated in f64 for the check."""
    lw = np.array([0.2126, 0.7152, 0.0722])
    amb = c0 * 0.282095
    g = np.array([c1x @ lw, c1y @ lw, c1z @ lw])
    gl = np.linalg.norm(g)
    if gl < 1e-6:
        return np.maximum(amb, 0), 0.0, 0.0
    d = g / gl
    dr = np.maximum(0.488603 * (c1x * d[0] + c1y * d[1] + c1z * d[2]), 0)
    x = n @ d
    if soft > 0:
        t = np.clip((x + soft) / (2 * soft), 0, 1)
        r = t * t * (3 - 2 * t)
    else:
        r = 1.0 if x > 0 else 0.0
    return np.maximum(amb - dr + 2 * dr * r, 0), float(x > 0), (dr @ lw) / max(amb @ lw, 1e-6)


def test_untagged_is_the_physical_gather():
    a, depth = _solve(None)
    b, _ = _solve(np.zeros((H, W), np.uint8))
    assert np.array_equal(a["irr"].view(np.uint32), b["irr"].view(np.uint32))
    alpha = a["irr"][..., 3]
    assert ((alpha == 1.0) == (depth > 0)).all() and ((alpha == 0.0) == (depth <= 0)).all()


def test_toon_pixels_go_through_the_receiving_operator():
    phys, depth = _solve(None)
    tag = np.zeros((H, W), np.uint8)
    tag[:, : W // 3] = 255            # toon
    tag[:, W // 3: 2 * W // 3] = 128  # another measured object
    got, _ = _solve(tag)
    fg = depth > 0
    alpha = got["irr"][..., 3]
    obj = fg.copy(); obj[:, : W // 3] = False; obj[:, 2 * W // 3:] = False
    pho = fg.copy(); pho[:, : 2 * W // 3] = False
    toon = fg.copy(); toon[:, W // 3:] = False
    assert (alpha[obj] == 2.0).all() and (alpha[pho] == 1.0).all()
    # object and photoreal pixels keep the physical irradiance
    assert np.array_equal(got["irr"][obj | pho][:, :3].view(np.uint32), phys["irr"][obj | pho][:, :3].view(np.uint32))
    # toon pixels: alpha 2 + band (+ 2), and the irradiance of toonReceive on the weighted L0 / L1
    lit = toon & (phys["irr"][..., :3].sum(-1) > 0)
    assert lit.sum() > 100
    assert set(np.unique(alpha[lit])) <= {2.0, 3.0, 4.0, 5.0}
    assert not np.array_equal(got["irr"][lit][:, :3], phys["irr"][lit][:, :3])
    assert (got["irr"][lit][:, :3] >= 0).all()


def test_receive_switch_keeps_the_physical_irradiance():
    """style.y = 0 (physical receiving): toon pixels keep the physical irradiance, their alpha still says toon."""
    phys, depth = _solve(None)
    tag = np.full((H, W), 255, np.uint8)
    got, _ = _solve(tag, style=(1.0, 0.0, 0.0))
    fg = depth > 0
    assert np.array_equal(got["irr"][fg][:, :3].view(np.uint32), phys["irr"][fg][:, :3].view(np.uint32))
    lit = fg & (phys["irr"][..., :3].sum(-1) > 0)
    assert (got["irr"][..., 3][lit] >= 2.0).all()


def test_toon_receive_formula():
    """The oracle's toonReceive against the formula in f64, on random SH and normals, hard and soft ramps."""
    rng = np.random.default_rng(7)
    for k in range(300):
        c = rng.normal(0.0, 1.0, 12).astype(np.float32)
        c[:3] = np.abs(c[:3]) * 3
        nn = rng.normal(0.0, 1.0, 3)
        nn = (nn / np.linalg.norm(nn)).astype(np.float32)
        soft = [0.0, 0.2, 0.5][k % 3]
        got = bind.toon_receive(c, nn, soft)
        c64 = c.astype(np.float64)
        e, band, contrast = _recv(c64[:3], c64[3:6], c64[6:9], c64[9:12], nn.astype(np.float64), soft)
        assert np.allclose(got[:3], e, rtol=1e-4, atol=1e-5), (k, got, e)
        if abs(nn.astype(np.float64) @ (np.array([c64[9:12], c64[3:6], c64[6:9]]) @ [0.2126, 0.7152, 0.0722])) > 1e-3:
            assert got[3] == band
        assert abs(got[4] - contrast) <= 1e-4 * max(1.0, abs(contrast))
    # no L1 gradient: the ambient alone
    got = bind.toon_receive(np.array([1, 2, 3] + [0] * 9, np.float32), np.array([0, 1, 0], np.float32), 0.0)
    assert np.allclose(got[:3], np.array([1, 2, 3]) * 0.282095) and got[3] == 0 and got[4] == 0
