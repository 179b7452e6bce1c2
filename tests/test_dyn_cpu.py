"""The oracle's dynamic layer (oracle/dyn.c, dynlayer.ts) against properties of its definition, on the CPU.

* the splat sums are fixed point, so the layer does not depend on the order of the dynamic triangles;
* the area words of level 0 add up to the sampled area of the triangles splatted there (each sample's trilinear weights
  sum to 1), within the rounding of the fixed-point adds;
* a level-1 voxel holds its own splats plus a quarter of each child (the resolve);
* bricks wanted last frame and not now are emptied, the frame counter advances and the bounds are published;
* a pool too small drops the finest bricks (ranks in bit order, coarse levels first), and a read there falls back to the
  coarser level;
* a ray through a closed box is covered, one that misses every box is not;
* log2 as the library defines it: exact at powers of two, within 2e-7 relative elsewhere."""
import dataclasses
import math

import numpy as np
import pytest

from oracle import bind
from rtgi import configs, frame as fr, movers, scenes

VOX = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}


@pytest.fixture(scope="module")
def world():
    base = scenes.room_scene(0, n_boxes=60)
    s, objs = movers.with_moving_boxes(base, 12, scenes.PCG32(3, stream=5), area=(0.0, 0.0, 4.0, 4.0), height=(0.3, 1.5))
    first = base.triangle_count
    v = configs.vox_params(VOX)
    st = bind.vox_build(dataclasses.replace(s, tri=s.tri[:first]), v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels,
                        s.camera.eye)
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=64, height=48, sun_dir=s.sun_dir, sun_e=fr.SUN_E, sky=fr.SKY))
    return s, objs, first, v, st, F


def _layer(s, st, first, F, nb=512):
    dl = bind.Dyn(st, nb)
    dl.build(s, st, first, s.triangle_count, F)
    return dl


def test_order_of_the_dynamic_triangles_does_not_matter(world):
    s, objs, first, v, st, F = world
    a = _layer(s, st, first, F)
    perm = np.random.default_rng(1).permutation(s.triangle_count - first) + first
    tri = s.tri.copy()
    tri[first:] = s.tri[perm]
    b = _layer(dataclasses.replace(s, tri=tri), st, first, F)
    for k in ("hdr", "ptr", "bits", "meta", "mask", "data"):
        assert np.array_equal(a.arrays[k], b.arrays[k]), k


def test_level0_area_is_the_sampled_area(world):
    s, objs, first, v, st, F = world
    dl = _layer(s, st, first, F)
    h = dl.arrays["hdr"]
    s0, n0 = int(h[16]), int(h[24])
    assert n0 > 0
    data = dl.arrays["data"].reshape(-1, 512, 13)[s0:s0 + n0]
    got = data[..., 6].astype(np.float64).sum() / 65536.0
    P = s.positions.astype(np.float64)
    lo = st["origin"][0, :3] * v.v0 * 8
    hi = lo + v.G * v.v0 * 8
    want, adds = 0.0, 0
    for t in range(first, s.triangle_count):
        a, b, c = (P[i] for i in s.tri[t, :3])
        mn, mx = np.minimum(np.minimum(a, b), c), np.maximum(np.maximum(a, b), c)
        if not ((mn - 2 * v.v0 > lo).all() and (mx + 2 * v.v0 < hi).all()):
            continue   # splatted at a coarser level
        want += 0.5 * np.linalg.norm(np.cross(b - a, c - a))
        e = max(np.linalg.norm(b - a), np.linalg.norm(c - b), np.linalg.norm(a - c))
        adds += 8 * max(1, min(16, math.ceil(e / v.v0))) ** 2
    want /= v.v0 ** 2
    assert abs(got - want) <= 0.5 / 65536 * adds + 1e-4 * want, (got, want)


def test_resolve_quarters_the_children(world):
    s, objs, first, v, st, F = world
    dl = _layer(s, st, first, F)
    a, h = dl.arrays, dl.arrays["hdr"]
    G, G3 = v.G, v.G ** 3
    data = a["data"].reshape(-1, 512, 13)
    org = st["origin"]
    checked = 0
    for slot in range(int(h[17]), int(h[17] + h[25])):      # level 1
        pi = int(a["meta"][slot])
        r = pi % G3
        for bit in range(512):
            if not (a["mask"][slot * 16 + bit // 32] >> (bit % 32)) & 1:
                continue
            c = np.array([r % G * 8 + (bit & 7), (r // G) % G * 8 + ((bit >> 3) & 7), r // (G * G) * 8 + (bit >> 6)])
            gc = (org[1, :3] * 8 + c) * 2 - org[0, :3] * 8
            cp = int(a["ptr"][((gc[2] >> 3) * G + (gc[1] >> 3)) * G + (gc[0] >> 3)])
            if cp >= dl.nb:
                continue
            kid = 0.0
            for q in range(8):
                l = (gc & 7) + np.array([q & 1, (q >> 1) & 1, q >> 2])
                kid += int(data[cp, l[0] + 8 * l[1] + 64 * l[2], 6]) / 65536.0
            val = float(data[slot, bit, 6:7].view(np.float32)[0])
            assert val >= 0.25 * kid * (1 - 1e-5) - 1e-6
            checked += 1
    assert checked > 50


def test_bricks_of_the_last_frame_are_emptied(world):
    s, objs, first, v, st, F = world
    dl = _layer(s, st, first, F)
    before = dl.arrays["ptr"].copy()
    h1 = dl.arrays["hdr"].copy()
    P, N = s.positions.copy(), s.normals.copy()
    P[objs.first:] += np.array([30.0, 0.0, 0.0], np.float32)   # every box far out of the windows
    dl.build(dataclasses.replace(s, positions=P, normals=N), st, first, s.triangle_count, F)
    h2 = dl.arrays["hdr"]
    assert h1[10] == 1 and h2[10] == 2
    assert h2[0] < h1[0]
    gone = (before < dl.nb) & (dl.arrays["ptr"] == 0xffffffff)
    assert gone.sum() > 0
    assert (h1[2:5] < h1[5:8]).all()                             # bounds published (cm + 2^30)


def test_pool_overflow_drops_the_finest_bricks(world):
    s, objs, first, v, st, F = world
    dl = _layer(s, st, first, F, nb=24)
    h, ptr = dl.arrays["hdr"], dl.arrays["ptr"]
    G3 = v.G ** 3
    assert h[1] > 0 and h[8] == 24 and h[0] == h[1] + h[8]
    # slots by rank in bit order, coarse levels first: the coarsest level keeps every brick, the finest loses some
    lvl = np.arange(ptr.size) // G3
    assert ((ptr[lvl == 2] < 24) | (ptr[lvl == 2] == 0xffffffff)).all()
    assert (ptr[lvl == 0] == 0xfffffffd).any()
    # a read where a level-0 brick was dropped falls back to the coarser level (which holds only its own splats)
    c = objs.centres[0]
    out = dl.trace(st, [c[0] - 3.0, c[1], c[2]], [1.0, 0.0, 0.0], 0.05, 6.0, 0.05)
    assert 0.0 <= out[3] <= 1.0


def test_rays_through_and_past_a_box(world):
    s, objs, first, v, st, F = world
    dl = _layer(s, st, first, F)
    c = objs.centres[0]
    hit = dl.trace(st, [c[0] - 3.0, c[1], c[2]], [1.0, 0.0, 0.0], 0.05, 6.0, 0.05)
    assert hit[3] == pytest.approx(1.0) and (hit[:3] >= 0).all()
    miss = dl.trace(st, [0.0, 3.9, 0.0], [0.0, 1.0, 0.0], 0.05, 2.0, 0.05)   # up from above every box
    assert miss[3] == 0.0


def test_log2_definition():
    for k in range(-20, 21):
        assert bind.log2(2.0 ** k) == k
    xs = np.random.default_rng(2).uniform(-30, 30, 20000)
    for x in 2.0 ** xs[:2000]:
        x = float(np.float32(x))
        assert abs(bind.log2(x) - math.log2(x)) <= 2e-7 * max(1.0, abs(math.log2(x)))


def test_objects_receive_the_bounce_volume(world):
    """The token obj (phase 31) in the oracle: from the second frame on, dynInject adds albedo / pi times the previous
    volume's irradiance to the layer's radiance words (level 0 in fixed point: never less than before); a layer without
    albedo words receives nothing; the volume's rays, which read the layer, then differ from a volume without it."""
    s, objs, first, v, st0, F = world
    bn = {"cell": 0.8, "dims": (16, 8, 16), "rays": 16, "div": 1}
    runs = {}
    for name, albedo, objects in (("obj", True, True), ("plain", True, False), ("no-albedo", False, True)):
        st = dict(st0)
        dl = bind.Dyn(st, 512, albedo=albedo)
        ob = bind.Bounce(st, objects=objects, **bn)
        grew = 0
        for f in range(2):
            dl.build(s, st, first, s.triangle_count, F)
            st["dyn"] = dl
            before = dl.arrays["data"].copy()
            ob.frame(st, F)
            after = dl.arrays["data"]
            if f == 0 or not objects or not albedo:
                assert np.array_equal(after, before), f"{name}, frame {f}: the layer changed"
            else:
                h = dl.arrays["hdr"]
                s0, n0 = int(h[16]), int(h[24])
                a = after.reshape(-1, 512, 13)[s0:s0 + n0, :, 7:10]
                b = before.reshape(-1, 512, 13)[s0:s0 + n0, :, 7:10]
                assert (a >= b).all(), "level 0 receives non-negative light (fixed point)"
                grew = int((a > b).sum())
        runs[name] = (grew, [x.copy() for x in ob.vol])
    assert runs["obj"][0] > 100
    # the volume's rays see the objects: its second volume differs from the one traced without the layer
    assert not np.array_equal(runs["obj"][1][1], runs["plain"][1][1])
