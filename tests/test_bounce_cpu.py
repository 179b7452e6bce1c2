"""The oracle's multi-bounce volume (bounce.ts) on the CPU: the direction table, and properties of a frame of the
volume over the leak room (the reference pins no output of it for a reproducible scene)."""
import numpy as np

import gi_cases
from oracle import bind


def test_bounce_dirs_cover_the_sphere():
    d = bind.bounce_dirs(16)
    assert d.shape == (16, 4) and d.dtype == np.float32
    assert np.allclose(np.linalg.norm(d[:, :3].astype(np.float64), axis=1), 1.0, atol=1e-6)
    assert np.allclose(d[:, 2], 1.0 - (2.0 * np.arange(16) + 1.0) / 16.0)   # z = 1 - (2i + 1) / n
    assert abs(d[:, :3].astype(np.float64).sum(axis=0)).max() < 0.2          # spread over the sphere


def _world(case):
    v = case.vox
    st = bind.vox_build(case.scene, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, case.scene.camera.eye)
    shadow = bind.shadow_render(case.scene, case.frame, case.shadow)
    bind.vox_sun(st, case.frame, shadow)
    return st


def test_bounce_frames_over_the_leak_room():
    case = gi_cases.leak_sun(0.1, "f32", 512)
    st = _world(case)
    b = bind.Bounce(st)
    nv = int(min(st["hdr"][1], case.vox.maxVoxels))
    inj1 = b.frame(st, case.frame)[: nv * 6].reshape(nv, 6)
    listed1 = int(b.list[0])
    assert listed1 > 0 and b.list[1] == 1 and b.list[2] == 1
    assert np.isfinite(inj1).all() and (inj1 >= 0).all()
    assert (inj1 > 0).mean() > 0.1          # sunlit walls and floor reflect into their neighbours
    # the origin texel of the current volume holds the probe coordinates of probe 0
    k = 6 * 32 * 16 * 32 * 4                 # texel (0, 0, 6 dz)
    o = b.vol[1][k:k + 3]
    eye = np.float32(case.scene.camera.eye)
    assert np.array_equal(o, np.floor(eye / np.float32(1.2)) - np.array([16, 8, 16], np.float32))
    # the second frame traces the other half of the probes (div 2) and reads the first volume in its rays
    inj2 = b.frame(st, case.frame)[: nv * 6].reshape(nv, 6)
    assert b.list[1] == 2 and b.list[2] == 0 and 0 < int(b.list[0]) < listed1 * 2
    assert (inj2 >= inj1 - 1e-3 * (1 + inj1)).mean() > 0.95   # a second bounce adds light
    assert inj2.sum() > inj1.sum()


def test_bounce_without_light_is_zero():
    case = gi_cases.leak_sun(0.1, "f32", 512)
    f = np.array(case.frame, np.float32).copy()
    f[92:95] = 0.0          # no sun
    f[96:99] = 0.0          # no sky
    st = _world(case)
    b = bind.Bounce(st)
    for _ in range(2):
        inj = b.frame(st, f)
        assert (inj == 0.0).all()
