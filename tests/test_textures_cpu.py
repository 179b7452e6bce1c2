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
