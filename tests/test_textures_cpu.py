"""Base colour textures in the oracle (oracle/tex.c; scene_gpu.ts:60-89, voxel.ts:325-336): the decode, the mip
chain, the bilinear repeat sampler, and their effect on the rebuild — alpha-masked texels cut voxels out of a panel,
sampled colours become the voxels' albedo."""
import dataclasses

import numpy as np

from oracle import bind
from rtgi import scenes


def _srgb(k):
    c = k / 255.0
    return np.float32(c / 12.92 if c <= 0.04045 else ((c + 0.055) / 1.055) ** 2.4)


def test_decode_and_mip_chain():
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, (2, 8, 8, 4), dtype=np.uint8)
    ch = bind.texture_chain(img)
    assert ch.shape == (2, 64 + 16 + 4 + 1, 4)
    l0 = ch[:, :64].reshape(2, 8, 8, 4)
    for k in range(256):
        m = img[..., :3] == k
        assert (l0[..., :3][m] == _srgb(k)).all()
    assert np.array_equal(l0[..., 3], (img[..., 3].astype(np.float32) / np.float32(255.0)))
    l1 = ch[:, 64:80].reshape(2, 4, 4, 4)
    want = ((l0[:, 0::2, 0::2] + l0[:, 0::2, 1::2]) + (l0[:, 1::2, 0::2] + l0[:, 1::2, 1::2])) * np.float32(0.25)
    assert np.array_equal(l1, want)
    assert np.allclose(ch[:, -1], l0.reshape(2, -1, 4).mean(1), rtol=1e-5)


def test_sampler_centres_midpoints_and_repeat():
    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, (1, 4, 4, 4), dtype=np.uint8)
    l0 = bind.texture_chain(img)[0, :16].reshape(4, 4, 4)
    for j in range(4):
        for i in range(4):
            u, v = (i + 0.5) / 4, (j + 0.5) / 4
            assert np.array_equal(bind.tex_sample(img, u, v, 0), l0[j, i])
            assert np.array_equal(bind.tex_sample(img, u + 3.0, v - 2.0, 0), l0[j, i])   # repeat
    mid = bind.tex_sample(img, 2.0 / 4, 0.5 / 4, 0)                      # between texels 1 and 2 of row 0
    assert np.allclose(mid, (l0[0, 1] + l0[0, 2]) / 2, atol=1e-6)
    edge = bind.tex_sample(img, 0.0, 0.5 / 4, 0)                        # wraps between texels 3 and 0
    assert np.allclose(edge, (l0[0, 3] + l0[0, 0]) / 2, atol=1e-6)
    top = bind.tex_sample(img, 0.3, 0.7, 9)                             # past the chain: the 1 x 1 level
    assert np.allclose(top, l0.reshape(-1, 4).mean(0), rtol=1e-5)


def _occupied(st):
    return sum(bin(int(w)).count("1") for w in st["occ"][: int(st["hdr"][0]) * 16])


def test_masked_panels_and_textured_albedo_in_the_rebuild():
    s = scenes.textured_scene()
    eye = s.camera.eye
    args = (0.08, 3, 16, 8192, 1 << 20, eye)
    tex = bind.vox_build(s, *args)
    # the same panels opaque (untextured, alpha 1): the lattice's holes are filled
    mats = [dataclasses.replace(m, base_color_tex=0) if m.name == "panel" else m for m in s.materials]
    opaque = bind.vox_build(dataclasses.replace(s, materials=mats), *args)
    assert _occupied(tex) < _occupied(opaque)
    # no texture at all: the alpha-masked panels keep every voxel, the boxes take the factor as albedo
    plain = bind.vox_build(dataclasses.replace(s, textures=None, uvs=None), *args)
    assert _occupied(plain) == _occupied(opaque)
    nv = int(tex["hdr"][1])
    alb = tex["attr"][0: nv * 4: 4]
    albp = plain["attr"][0: int(plain["hdr"][1]) * 4: 4]
    assert len(np.unique(alb & 0xffffff)) > len(np.unique(albp & 0xffffff))


def test_rasters_cut_the_holes():
    """The G-buffer and the shadow map leave out masked fragments: the lattice panels' holes show what is behind
    them; an untextured masked material whose factor's alpha is below the cutoff draws nothing at all."""
    from rtgi import frame as fr
    s = scenes.textured_scene()
    W, H = 160, 120
    bmin, bmax = fr.scene_bounds(s.positions)
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, cascades=2,
                                     light_view_proj=fr.scene_sun_view_proj(bmin, bmax, s.sun_dir),
                                     shadow_bias=fr.SHADOW_BIAS))
    solid = dataclasses.replace(s, textures=None, uvs=None)
    d_tex, _, tri_tex = bind.raster_gbuffer(s, F, W, H)
    d_solid, _, tri_solid = bind.raster_gbuffer(solid, F, W, H)
    panel = len(s.materials) - 1
    on_panel = lambda tri: (tri != 0xffffffff) & (s.tri[np.where(tri == 0xffffffff, 0, tri), 3] == panel)
    assert on_panel(tri_solid).sum() > on_panel(tri_tex).sum() > 0
    m_tex, m_solid = bind.shadow_render(s, F, 256), bind.shadow_render(solid, F, 256)
    assert (m_tex != m_solid).any() and (m_tex >= m_solid).all()   # holes let the depth fall back further
    clear = [dataclasses.replace(m, base_color=(0.9, 0.9, 0.9, 0.2)) if m.name == "panel" else m for m in s.materials]
    gone = dataclasses.replace(solid, materials=clear)
    _, _, tri_gone = bind.raster_gbuffer(gone, F, W, H)
    assert on_panel(tri_gone).sum() == 0


def test_world_clusters_carry_uvs():
    """with_world's clustered vertices take the uv of the member vertex nearest their mean (world.ts:124, 137)."""
    from rtgi import world as W
    s = scenes.textured_scene()
    s2, w = W.with_world(s, [(0, 0, 0), (12, 0, 0)], 0.08, 3)
    assert s2.uvs.shape == (s2.positions.shape[0], 2)
    assert np.array_equal(s2.uvs[: s.positions.shape[0]], s.uvs)
    extra = s2.uvs[s.positions.shape[0]:]
    assert len(extra) > 0 and set(map(tuple, extra)) <= set(map(tuple, s.uvs))
