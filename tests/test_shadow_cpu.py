"""The oracle's sun shadow map and voxel sun visibility (lighting.ts:100-106, 133-189; frame.ts:35-52; voxel.ts:633-671)
against known answers on a scene whose shadow is known in closed form."""
import numpy as np

from oracle import bind
from rtgi import frame as fr, mathx, scenes


def _scene(sun_dir=(0.0, 1.0, 0.0)):
    """A 10 x 10 m ground at y = 0 and a 2 x 1 x 2 m box floating at y in [1, 2] over the origin."""
    b = scenes.Builder([scenes.Material("grey", (0.5, 0.5, 0.5, 1.0))])
    b.quad([-5, 0, 5], [5, 0, 5], [5, 0, -5], [-5, 0, -5])
    b.box((0.0, 1.5, 0.0), (1.0, 0.5, 1.0))
    return b.scene("shadow-ks", scenes.Camera((0, 3, 6), (0, 0, 0), 60, 0.05), sun_dir=sun_dir)


def _frame(s, S):
    bmin, bmax = fr.scene_bounds(s.positions)
    lvp = fr.scene_sun_view_proj(bmin, bmax, s.sun_dir)
    return fr.pack_frame(fr.FrameParams(cam=s.camera, width=64, height=64, sun_dir=s.sun_dir, light_view_proj=lvp,
                                        shadow_bias=fr.SHADOW_BIAS, cascades=2))


def test_sun_view_proj_is_the_reference_formula():
    """sceneSunViewProj: the bounding sphere's sunward pole at depth 0, its centre at 0.5, the far pole at 1."""
    s = _scene((0.3, 1.0, 0.2))
    bmin, bmax = fr.scene_bounds(s.positions)
    m = np.array(fr.scene_sun_view_proj(bmin, bmax, s.sun_dir), np.float64).reshape(4, 4).T
    c = (np.array(bmin) + np.array(bmax)) / 2
    r = mathx.hypot(*(np.array(bmax) - np.array(bmin))) / 2
    d = np.array(s.sun_dir) / np.linalg.norm(s.sun_dir)
    for p, z in ((c + d * r, 0.0), (c, 0.5), (c - d * r, 1.0)):
        q = m @ np.array([*p, 1.0])
        assert abs(q[2] - z) < 1e-5 and abs(q[3] - 1.0) < 1e-6
        assert abs(q[0]) < 1e-5 and abs(q[1]) < 1e-5   # on the light axis: the map centre


def test_shadow_map_known_answer():
    s = _scene()
    S = 256
    F = _frame(s, S)
    m = bind.shadow_render(s, F, S)
    lvp = np.array(F[64:80], np.float64).reshape(4, 4).T
    zbox = (lvp @ np.array([0, 2, 0, 1.0]))[2]
    zground = (lvp @ np.array([3, 0, 3, 1.0]))[2]
    assert zbox < zground
    # texels under the box hold its top face, texels over the bare ground the ground, nothing drawn beyond the scene
    def texel(x, z):
        q = lvp @ np.array([x, 0.0, z, 1.0])
        u, v = q[0] * 0.5 + 0.5, q[1] * -0.5 + 0.5
        return int(v * S), int(u * S)
    assert abs(m[texel(0.2, 0.3)] - zbox) < 1e-3
    assert abs(m[texel(3.0, -3.5)] - zground) < 1e-3
    assert (m <= 1.0).all() and (m == 1.0).any() and (m < 1.0).mean() > 0.3
    # the bias is positive and small: a stored depth sits just behind its surface
    assert 0.0 < m[texel(3.0, -3.5)] - zground < 1e-3


def test_shadow_map_does_not_depend_on_triangle_order():
    s = _scene((0.3, 1.0, 0.2))
    F = _frame(s, 128)
    m1 = bind.shadow_render(s, F, 128)
    perm = np.random.default_rng(3).permutation(s.tri.shape[0])
    s2 = scenes.Scene(s.name, s.positions, s.normals, s.tri[perm].copy(), s.materials, s.camera, s.sun_dir)
    m2 = bind.shadow_render(s2, F, 128)
    assert np.array_equal(m1.view(np.uint32), m2.view(np.uint32))


def test_sun_tap_known_answer():
    s = _scene()
    S = 512
    F = _frame(s, S)
    m = bind.shadow_render(s, F, S)
    assert bind.sun_tap(F, m, [0.0, 0.03, 0.0]) == 0.0      # under the box
    assert bind.sun_tap(F, m, [0.5, 0.5, -0.4]) == 0.0      # between the box and the ground
    assert bind.sun_tap(F, m, [3.5, 0.03, 3.5]) == 1.0      # open ground
    assert bind.sun_tap(F, m, [0.0, 2.03, 0.0]) == 1.0      # on the box
    assert bind.sun_tap(F, m, [0.0, 0.03, 40.0]) == 1.0     # outside the map: lit
    # across the shadow's edge (x = 1) the comparison is filtered over two texels
    xs = np.linspace(0.9, 1.1, 41)
    v = np.array([bind.sun_tap(F, m, [x, 0.03, 0.0]) for x in xs])
    assert v[0] == 0.0 and v[-1] == 1.0 and (np.diff(v) >= 0).all() and ((v > 0) & (v < 1)).any()


def test_voxel_sun_visibility_known_answer():
    """voxSun over the voxelised scene: ground voxels in the box's shadow 0, open ground and the box's top 1."""
    s = _scene()
    S = 512
    F = _frame(s, S)
    m = bind.shadow_render(s, F, S)
    st = bind.vox_build(s, 0.1, 1, 16, 4096, 1 << 18, (0.0, 1.0, 0.0))
    bind.vox_sun(st, F, m)
    nb, nv = int(st["hdr"][0]), int(st["hdr"][1])
    assert nb > 0 and nv > 0
    # voxel centres in attribute order (resolveAttr's rank order within each brick)
    cent = np.zeros((nv, 3))
    org = st["origin"][0, :3]
    for b in range(nb):
        code, first = int(st["code"][b]), int(st["base"][b])
        bx, by, bz = (code >> 18) & 511, (code >> 9) & 511, code & 511
        r = 0
        for bit in range(512):
            if st["occ"][b * 16 + (bit >> 5)] >> (bit & 31) & 1:
                c = np.array([bx * 8 + (bit & 7), by * 8 + ((bit >> 3) & 7), bz * 8 + (bit >> 6)])
                cent[first + r] = (org * 8 + c + 0.5) * 0.1
                r += 1
    vis = st["sunvis"][:nv]
    ground = cent[:, 1] < 0.1
    under = ground & (np.abs(cent[:, 0]) < 0.8) & (np.abs(cent[:, 2]) < 0.8)
    open_ = ground & ((np.abs(cent[:, 0]) > 1.3) | (np.abs(cent[:, 2]) > 1.3))
    top = (cent[:, 1] > 1.9) & (np.abs(cent[:, 0]) < 0.8) & (np.abs(cent[:, 2]) < 0.8)
    assert under.any() and open_.any() and top.any()
    assert (vis[under] == 0.0).all()
    assert (vis[open_] == 1.0).all()
    assert (vis[top] == 1.0).all()


def test_js_round_is_math_round():
    """Math.round: halves toward +infinity, and no double rounding below one half."""
    assert fr._js_round(0.49999999999999994) == 0.0 and fr._js_round(0.5) == 1.0
    assert fr._js_round(-2.5) == -2.0 and fr._js_round(2.5) == 3.0 and fr._js_round(-0.6) == -1.0


def test_camera_following_layers():
    """cameraMatrix (lighting.ts:115-123): layer 0 of half width 32 m and layer 1 of 410 m centred on the camera's
    position across the sun, snapped to the layer's texels, depth 0.5 at the camera; moving the camera less than a
    texel across the sun leaves the lateral placement where it was."""
    sun = (0.3, 1.0, 0.2)
    eye = (13.37, 1.6, -7.21)
    S = 4096
    near, far = fr.world_sun_view_projs(sun, eye, S)
    for m, r in ((near, fr.SHADOW_NEAR_R), (far, fr.SHADOW_FAR_R)):
        M = np.array(m, np.float64).reshape(4, 4).T
        q = M @ np.array([*eye, 1.0])
        texel_ndc = 2.0 / S
        assert abs(q[0]) <= 0.5 * texel_ndc + 1e-6 and abs(q[1]) <= 0.5 * texel_ndc + 1e-6   # centred within a texel
        assert abs(q[2] - 0.5) < 1e-5
        d = np.array(sun) / np.linalg.norm(sun)
        assert abs((M @ np.array([*(np.array(eye) + d * fr.SHADOW_DEPTH_R), 1.0]))[2]) < 1e-4
        x = np.array(eye) + np.cross(d, [0, 1.0, 0]) / np.linalg.norm(np.cross(d, [0, 1.0, 0])) * (r * 0.999)
        assert abs(abs((M @ np.array([*x, 1.0]))[0]) - 0.999) < 1e-3 or abs(abs((M @ np.array([*x, 1.0]))[1]) - 0.999) < 1e-3
    # the snapped placement: a step of a tenth of a layer-0 texel across the sun keeps x/y translation
    t0 = 2 * fr.SHADOW_NEAR_R / S
    up0 = np.array([0, 1.0, 0])
    right = np.cross(up0, np.array(sun) / np.linalg.norm(sun))
    right /= np.linalg.norm(right)
    e2 = tuple(np.array(eye) + right * (0.1 * t0))
    n2, _ = fr.world_sun_view_projs(sun, e2, S)
    snap = lambda e: fr._js_round(float(np.dot(e, right)) / t0)
    if snap(eye) == snap(e2):
        assert n2[12] == near[12] and n2[13] == near[13]


def _world_frame(s, S, eye):
    near, far = fr.world_sun_view_projs(s.sun_dir, eye, S)
    return fr.pack_frame(fr.FrameParams(cam=s.camera, width=64, height=64, sun_dir=s.sun_dir, light_view_proj=near,
                                        shadow_far=far, shadow_bias=fr.SHADOW_WORLD_BIAS, cascades=2))


def test_two_layer_tap_picks_the_layer():
    """shadowCoord with two layers: a point inside layer 0 reads layer 0; a point outside it reads layer 1 as a
    one-layer frame made of layer 1 would; outside both it is lit.  The layers are drawn from their own matrices."""
    b = scenes.Builder([scenes.Material("grey", (0.5, 0.5, 0.5, 1.0))])
    b.quad([-300, 0, 300], [300, 0, 300], [300, 0, -300], [-300, 0, -300])
    b.box((0.0, 1.5, 0.0), (1.0, 0.5, 1.0))     # a box near the camera
    b.box((100.0, 1.5, 0.0), (8.0, 0.5, 8.0))   # a wide one 100 m away (layer 1 only: 1.6 m texels at 512^2)
    s = b.scene("layers", scenes.Camera((0, 3, 6), (0, 0, 0), 60, 0.05), sun_dir=(0.0, 1.0, 0.0))
    S = 512
    F = _world_frame(s, S, (0.0, 1.6, 0.0))
    assert int(F[156]) == 2
    m = bind.shadow_render(s, F, S)
    assert m.shape == (2, S, S) and (m[0] < 1).any() and (m[1] < 1).any()
    # layer 1 alone, as a one-layer frame: the same map and the same taps outside layer 0
    F1 = F.copy()
    F1[64:80] = F[140:156]
    F1[156:159] = [1, F[158], 0]
    m1 = bind.shadow_render(s, F1, S)
    assert np.array_equal(m1.view(np.uint32), m[1].view(np.uint32))
    assert bind.sun_tap(F, m, [0.0, 0.03, 0.0]) == 0.0          # under the near box: layer 0
    far_pt = [100.0, 0.03, 0.0]                                 # under the far box: outside layer 0, inside layer 1
    assert bind.sun_tap(F, m, far_pt) == bind.sun_tap(F1, m1, far_pt) == 0.0
    assert bind.sun_tap(F, m, [100.0, 0.03, 30.0]) == 1.0
    assert bind.sun_tap(F, m, [0.0, 0.03, 900.0]) == 1.0        # outside both layers
    F_one = F.copy()
    F_one[156] = 1                                              # one layer: the far box's shadow is not seen
    assert bind.sun_tap(F_one, m, far_pt) == 1.0
