"""CPU-only checks: the C-ABI library loads and exports every symbol include/gi.h declares, the host mirror of the
reference's frame math and config grammar, and the oracle's builtins against their specifications."""
import ctypes as C
import math
import os
import re
from fractions import Fraction

import numpy as np
import pytest

from oracle import bind
from rtgi import _lib, configs, frame as fr, mathx, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "gi.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(gi_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in gi.h but not exported"
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"
    assert set(_lib.SIGNATURES) == set(syms)
    assert lib.gi_version() == 1
    assert lib.gi_status_string(-1) == b"invalid argument"


def test_no_device_is_an_error_not_a_fallback():
    # without a GPU the context cannot be made; the call returns a status, it does not run anything on the CPU
    lib = _lib.load()
    h = C.c_void_p()
    st = lib.gi_ctx_create(0, C.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        assert st == 0
        lib.gi_ctx_destroy(h)
    else:
        assert st in (_lib.GI_ERR_CUDA, _lib.GI_ERR_INVALID)
        assert lib.gi_last_error()


def test_null_arguments_are_rejected():
    lib = _lib.load()
    assert lib.gi_ctx_create(0, None) == _lib.GI_ERR_INVALID
    assert lib.gi_vox_build(None, None) == _lib.GI_ERR_INVALID
    assert b"NULL" in lib.gi_last_error()
    assert lib.gi_rc_solve(None, None, None) == _lib.GI_ERR_INVALID


def test_parse_config_grammar():
    p = configs.parse_config("screen-8-voxel-rc2-vs0.5-vo2-vk0.25-l2-dda64-bf16")
    assert (p.method, p.P, p.world, p.depthCascades, p.resCap) == ("screen", 8, "voxel", 0, 2)
    assert (p.voxScale, p.voxOffset, p.voxSkip, p.levelMap, p.ddaCap, p.atlas) == (0.5, 2.0, 0.25, 2, 64, "bf16")
    assert configs.parse_config("world-32").world == "none"
    assert configs.parse_config("screen-8-hybrid").depthCascades == 1
    with pytest.raises(ValueError, match="unknown config token"):
        configs.parse_config("screen-8-bogus")
    with pytest.raises(ValueError, match="unknown voxel parameter"):
        configs.vox_params({"v1": 0.1})
    assert configs.vox_params({"G": 16}).G == 16 and configs.DEFAULT_VOX.G == 32


def test_cascade_layout_config1():
    p = configs.parse_config("screen-8-voxel", {"cascades": 5})
    lay = configs.cascade_layout(p, 1920, 1080)
    tiles = [(c["tiles_x"], c["tiles_y"]) for c in lay["casc"]]
    assert tiles == [(240, 135), (120, 68), (60, 34), (30, 17), (15, 9)]
    assert [c["res"] for c in lay["casc"]] == [4, 8, 16, 32, 64]
    assert [(c["b0"], c["b1"]) for c in lay["casc"]][:3] == [(0.0, 1.0), (1.0, 5.0), (5.0, 21.0)]
    assert lay["rays_total"] == 2638080


def test_v8_hypot_and_matrices():
    assert mathx.hypot(3, 4) == 5.0
    assert mathx.hypot(0, 0, 0) == 0.0
    cam = fr.Camera((2.6, 1.6, 1.8), (0.2, 1.0, -1.4), 75, 0.05)
    m = fr.camera_matrices(cam, 1920, 1080)
    vp = np.array(m["viewProj"], np.float64).reshape(4, 4).T
    ivp = np.array(m["invViewProj"], np.float64).reshape(4, 4).T
    assert np.allclose(vp @ ivp, np.eye(4), atol=1e-5)
    # the near plane maps to depth 1, the eye looks along fwd
    p = np.array([*np.add(cam.eye, np.multiply(m["fwd"], 0.05)), 1.0])
    c = vp @ p
    assert abs(c[2] / c[3] - 1.0) < 1e-4


def test_pack_frame_layout():
    cam = fr.Camera((1.0, 2.0, 3.0), (0.0, 2.0, 0.0), 60, 0.1)
    F = fr.pack_frame(fr.FrameParams(cam=cam, width=640, height=360, cascades=3, P=8, sun_dir=(0, 2, 0)))
    u = F.view(np.uint32)
    assert F.size == 160 and F.dtype == np.float32
    assert list(F[80:84]) == [1.0, 2.0, 3.0, np.float32(0.1)]
    assert list(F[88:91]) == [0.0, 1.0, 0.0]
    assert list(F[100:104]) == [640, 360, np.float32(1 / 640), np.float32(1 / 360)]
    assert F[105] == np.float32(2 * math.tan(math.pi / 6) / 360)
    assert u[112] == 3
    assert abs(F[120:136].sum() - 4 * math.pi) < 1e-4   # octSolidAngles covers the sphere


def test_oct_solid_angles_symmetry():
    w = fr.oct_solid_angles(4)
    assert np.allclose(w.reshape(4, 4), w.reshape(4, 4)[::-1, ::-1], rtol=1e-3)
    assert abs(w.sum() - 4 * math.pi) < 1e-4


def test_pack_builtins_known_answers():
    lib = bind.lib()
    # WGSL: pack4x8unorm(e) = floor(0.5 + 255 * clamp(e, 0, 1)) per byte, x lowest
    v = (C.c_float * 4)(0.0, 1.0, 0.5, 2.0)
    assert lib.orc_pack4x8unorm(v) == (0 | (255 << 8) | (128 << 16) | (255 << 24))
    # pack2x16snorm: floor(0.5 + 32767 * clamp(e, -1, 1)) as i16
    assert lib.orc_pack2x16snorm(1.0, -1.0) == (32767 | ((-32767 & 0xffff) << 16))
    assert lib.orc_pack2x16snorm(0.0, -0.5) == (0 | ((-16383 & 0xffff) << 16))


def test_f16_bf16_conversions_match_numpy():
    lib = bind.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.standard_normal(2000) * 10, rng.standard_normal(500) * 1e-5, [65504, 65520, 1e6, -0.0, 6e-8]]).astype(np.float32)
    for x in xs:
        h = lib.orc_f32_to_f16(float(x))
        assert h == np.float16(x).view(np.uint16), x
        assert lib.orc_f16_to_f32(h) == np.float32(np.float16(x)) or math.isnan(x)


def _sat_exact(c, h, a, b, cc):
    """Separating-axis test in exact rationals: does the closed box (c, h) meet the triangle?"""
    F = lambda v: [Fraction(float(x)) for x in v]
    c, h, a, b, cc = F(c), F(h), F(a), F(b), F(cc)
    v = [[a[i] - c[i] for i in range(3)], [b[i] - c[i] for i in range(3)], [cc[i] - c[i] for i in range(3)]]
    e = [[v[1][i] - v[0][i] for i in range(3)], [v[2][i] - v[1][i] for i in range(3)], [v[0][i] - v[2][i] for i in range(3)]]
    axes = [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
    cr = lambda p, q: [p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]]
    axes.append(cr(e[0], e[1]))
    for ei in e:
        for u in ([1, 0, 0], [0, 1, 0], [0, 0, 1]):
            axes.append(cr(u, ei))
    for ax in axes:
        p = [sum(vi[k] * ax[k] for k in range(3)) for vi in v]
        r = sum(h[k] * abs(ax[k]) for k in range(3))
        if min(p) > r or max(p) < -r:
            return False
    return True


def test_tri_box_against_exact_separating_axes():
    lib = bind.lib()
    rng = np.random.default_rng(7)
    agree = 0
    n = 3000
    for _ in range(n):
        c = rng.uniform(-1, 1, 3).astype(np.float32)
        h = np.full(3, rng.uniform(0.05, 0.5), np.float32)
        tri = (c + rng.uniform(-1, 1, (3, 3)) * rng.uniform(0.1, 2.0)).astype(np.float32)
        args = [np.ascontiguousarray(x, np.float32) for x in (c, h, tri[0], tri[1], tri[2])]
        got = lib.orc_tri_box(*[x.ctypes.data for x in args])
        agree += int(bool(got) == _sat_exact(*args))
    assert agree >= n - 3   # f32 rounding may flip grazing contacts only


def test_round_log2_exact():
    lib = bind.lib()
    for x in [1.0, 1.4142135, 1.4142137, 0.7071067, 0.7071068, 3.0, 0.1, 1e-3, 1234.5]:
        r = np.int32(np.uint32(lib.orc_round_log2(x)))
        assert r == round(math.log2(np.float32(x))), x


def test_scenes_shapes():
    s = scenes.room_scene(0)
    assert s.triangle_count == 12 + 2 + 200 * 12
    assert s.tri[:, 3].max() < len(s.materials)
    c = scenes.colonnade_scene(0)
    assert 255_000 < c.triangle_count < 265_000
    assert scenes.leak_room(0.1).triangle_count == 1212
    # Builder quads: face normal = normalize(cross(b - a, c - a)) per vertex
    n = s.normals[s.tri[0, 0]]
    assert abs(np.linalg.norm(n) - 1) < 1e-6


def test_f32out_token_and_layout():
    p = configs.parse_config("screen-8-voxel-f16-f32out-dda256", {"cascades": 3})
    assert p.atlas == "f16" and p.f32Out
    assert configs.cascade_layout(p, 64, 32)["f32_out"] == 1
    assert configs.cascade_layout(configs.parse_config("screen-8-voxel-f16"), 64, 32)["f32_out"] == 0


def test_irr16_token_and_the_oracle_store():
    """irr16: the irradiance rounded to rgba16float at the store (round to nearest even), nothing before it changed."""
    p = configs.parse_config("screen-8-voxel-f32-irr16", {"cascades": 3})
    assert p.atlas == "f32" and p.irr16 and not p.f32Out
    assert configs.cascade_layout(p, 64, 32)["irr_f16"] == 1
    assert configs.cascade_layout(configs.parse_config("screen-8-voxel-f32"), 64, 32)["irr_f16"] == 0
    s = scenes.room_scene(0)
    W, H = 96, 64
    v = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    st = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye)
    outs = []
    for name in ("screen-8-voxel-f32", "screen-8-voxel-f32-irr16"):
        q = configs.parse_config(name, {"cascades": 3})
        F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=fr.SUN_E,
                                         sky=fr.SKY, cascades=q.cascades, P=q.P))
        depth, normal, _ = bind.raster_gbuffer(s, F, W, H)
        outs.append(bind.rc_solve(st, configs.cascade_layout(q, W, H), F, depth, normal.astype(np.float16).astype(np.float32)))
    wide, narrow = outs
    assert np.array_equal(wide["rad"].view(np.uint32), narrow["rad"].view(np.uint32))
    assert (wide["irr"] > 0).any()
    assert np.array_equal(wide["irr"].astype(np.float16).astype(np.float32).view(np.uint32), narrow["irr"].view(np.uint32))


def test_quotient_shortcuts_of_the_shading_are_exact():
    """The hit shading replaces two f32 divisions by f64 products rounded to f32: k / 32767 for every 16-bit k (the
    snorm normal) and a / pi for the 256 albedo bytes a = k / 255.  Both equal the IEEE f32 quotients everywhere."""
    x = np.arange(-32768, 32768).astype(np.float32)
    q = x / np.float32(32767)
    alt = (x.astype(np.float64) * (1.0 / 32767.0)).astype(np.float32)
    assert np.array_equal(q.view(np.uint32), alt.view(np.uint32))
    a = np.arange(256).astype(np.float32) / np.float32(255)
    pi = np.float32(3.14159265)
    assert np.array_equal((a / pi).view(np.uint32),
                          (a.astype(np.float64) * (1.0 / np.float64(pi))).astype(np.float32).view(np.uint32))


def _round_f32(x: Fraction) -> np.float32:
    """x rounded to the nearest f32, ties to even (exact: the f64 guess and its neighbours compared as fractions)."""
    c = np.float32(float(x))
    best = None
    for y in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        d = abs(Fraction(float(y)) - x)
        if best is None or d < best[0] or (d == best[0] and int(y.view(np.uint32)) % 2 == 0):
            best = (d, y)
    return best[1]


def test_snorm16_by_corrected_reciprocal_is_the_quotient():
    """The hit shading decodes a snorm16 half as q = k * r, e = fma(-q, 32767, k), fma(e, r, q) with r = RN(1 / 32767)
    (two fused multiply-adds instead of a division): equal to the IEEE f32 quotient k / 32767 for all 65536 k.  Every
    step is evaluated exactly and rounded once, as the fused operations do."""
    r = np.float32(1.0) / np.float32(32767.0)
    fr, f32767 = Fraction(float(r)), Fraction(32767)
    x = np.arange(-32768, 32768).astype(np.float32)
    want = x / np.float32(32767.0)
    for k, w in zip(x, want):
        fk = Fraction(float(k))
        q = _round_f32(fk * fr)
        e = _round_f32(-Fraction(float(q)) * f32767 + fk)
        got = _round_f32(Fraction(float(e)) * fr + Fraction(float(q)))
        assert got.view(np.uint32) == w.view(np.uint32), int(k)
    # the albedo / pi table the shading reads: (k / 255) / pi as f32 quotients, the numbers the f64 products give
    a = np.arange(256).astype(np.float32) / np.float32(255)
    assert np.array_equal((a / np.float32(3.14159265)).view(np.uint32),
                          (a.astype(np.float64) * (1.0 / np.float64(np.float32(3.14159265)))).astype(np.float32).view(np.uint32))


def test_floor_div_clamp_bound():
    """The DDA takes clamp(floor(x / vs)) from q = x * RN(1 / vs) when the clamped floors of q -+ thr agree, thr =
    |q| 2^-20 + 2^-20, else from the quotient.  The bound it rests on: the IEEE quotient lies within [q - thr, q + thr]
    (the ends rounded to f32).  Checked over random x of every magnitude and every level size of the clipmaps here."""
    rng = np.random.default_rng(5)
    for v0 in (0.05, 0.08, 0.1, 0.16, 0.2, 0.25, 0.3):
        for L in range(8):
            vs = np.float32(np.ldexp(np.float32(v0), L))
            ivs = np.float32(1.0) / vs
            x = (rng.uniform(-1.0, 1.0, 200000) * rng.choice([1e-6, 1e-2, 1.0, 1e2, 1e3, 3e4], 200000)).astype(np.float32)
            q = x * ivs
            thr = np.abs(q) * np.float32(2.0 ** -20) + np.float32(2.0 ** -20)
            exact = x / vs
            assert ((exact >= q - thr) & (exact <= q + thr)).all()


def test_gi_exp_accuracy():
    """The weights' e^x (Cody-Waite reduction, degree-7 Horner polynomial with fused multiply-adds): relative error
    against the exact exponential below 3e-7 on [-80, 0] (the range -20 rel takes) and 0 below -80."""
    lib = bind.lib()
    xs = np.concatenate([np.linspace(-80.0, 0.0, 20001), -np.logspace(-8, 0, 2001)]).astype(np.float32)
    got = np.array([lib.orc_gi_exp(float(x)) for x in xs], np.float64)
    exact = np.exp(xs.astype(np.float64))
    rel = np.abs(got - exact) / exact
    assert rel.max() < 3e-7, rel.max()
    assert lib.orc_gi_exp(-80.5) == 0.0 and lib.orc_gi_exp(0.0) == 1.0


def _sat_axes(v, h, reduced):
    """The nine edge-axis tests of the triangle/box overlap in numpy f32, per row: the reference's three-term dot
    products, or the kernels' two-term form without the zero component."""
    f = np.float32
    v0, v1, v2 = v[:, 0], v[:, 1], v[:, 2]
    e = [v1 - v0, v2 - v1, v0 - v2]
    ok = np.ones(len(v), bool)
    for k in range(3):              # axis (1,0,0) x e, (0,1,0) x e, (0,0,1) x e
        for ei in e:
            a = np.zeros_like(ei)
            i, j = [(1, 2), (0, 2), (0, 1)][k]
            if k == 0:
                a[:, 1], a[:, 2] = -ei[:, 2], ei[:, 1]
            elif k == 1:
                a[:, 0], a[:, 2] = ei[:, 2], -ei[:, 0]
            else:
                a[:, 0], a[:, 1] = -ei[:, 1], ei[:, 0]
            if reduced:
                p = [vi[:, i] * a[:, i] + vi[:, j] * a[:, j] for vi in (v0, v1, v2)]
                r = h[:, i] * np.abs(a[:, i]) + h[:, j] * np.abs(a[:, j])
            else:
                p = [(vi[:, 0] * a[:, 0] + vi[:, 1] * a[:, 1]) + vi[:, 2] * a[:, 2] for vi in (v0, v1, v2)]
                r = (h[:, 0] * np.abs(a[:, 0]) + h[:, 1] * np.abs(a[:, 1])) + h[:, 2] * np.abs(a[:, 2])
            lo = np.minimum(np.minimum(p[0], p[1]), p[2])
            hi = np.maximum(np.maximum(p[0], p[1]), p[2])
            ok &= ~((lo > r) | (hi < -r))
            assert all(x.dtype == f for x in p)
    return ok


def test_sat_edge_axes_without_zero_terms_decide_the_same():
    """The kernels' edge-axis tests drop each axis's zero component; on random, axis-aligned and grid-snapped
    triangles against voxel boxes they decide exactly as the three-term form."""
    rng = np.random.default_rng(11)
    n = 400000
    c = (np.floor(rng.uniform(-50, 50, (n, 1, 3))) * 0.1 + 0.05).astype(np.float32)
    tri = rng.uniform(-0.3, 0.3, (n, 3, 3)).astype(np.float32)
    snap = rng.random(n) < 0.5      # vertices on the 0.05 grid: many zero edges and products
    tri[snap] = (np.round(tri[snap] / 0.05) * 0.05).astype(np.float32)
    flat = rng.integers(0, 3, n)    # axis-aligned triangles
    tri[np.arange(n), :, flat] = tri[np.arange(n), :1, flat]
    v = (c + tri).astype(np.float32) - c
    h = np.full((n, 3), np.float32(0.05 * 1.0001), np.float32)
    full, red = _sat_axes(v, h, False), _sat_axes(v, h, True)
    assert np.array_equal(full, red)
    assert 0.05 < full.mean() < 0.95
