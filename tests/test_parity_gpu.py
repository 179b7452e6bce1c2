"""Parity of the CUDA path (through the C-ABI) with the oracle, on the same inputs.

Bar: voxel state, G-buffer and DDA hit cells bit-exact; traced radiance, merged atlas and irradiance within 1e-4
relative in f32.  Every f32 step is reproducible (no fused multiply-add on either side, the weights' exp is the
library's own), so the test requires bit-exact outputs and reports the relative error when they differ."""
import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.destroy()


def _tol(atlas):
    return {"f32": 1e-4, "f16": 2.0 ** -10, "bf16": 2.0 ** -7}[atlas]


def _close(a, b, rel, what):
    """Bit-exact (the path has no implementation-defined f32 step left); the tolerance only words the report."""
    a32, b32 = np.asarray(a, np.float32), np.asarray(b, np.float32)
    if np.array_equal(a32.view(np.uint32), b32.view(np.uint32)):
        return
    a = a32.astype(np.float64)
    b = b32.astype(np.float64)
    bad = (a32.view(np.uint32) != b32.view(np.uint32))
    within = not (np.abs(a - b) > rel * np.abs(b) + 1e-6).any()
    assert False, f"{what}: {bad.sum()} of {bad.size} not bit-exact (within {rel:g} relative: {within}); first " \
                  f"{np.argwhere(bad)[:3].tolist()} gpu {a[bad][:3]} oracle {b[bad][:3]}"


def run_gpu(ctx, case, debug=True):
    sg = gpu.SceneGpu(ctx, case.scene)
    if case.movers:   # pose the moving objects on the device, as the serving loop does
        objs, t = case.movers
        sg.rigid_define(objs.first, objs.per, objs.centres.shape[0])
        sg.rigid_upload(objs.transforms(t))
        sg.rigid_apply()
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    rc.set_frame(case.frame)
    rc.render_gbuffer(sg)
    if case.shadow:
        rc.render_shadow(sg, case.shadow)
    vw.update(case.scene.camera.eye)
    rc.set_debug_hits(debug)
    rc.solve(vw)
    res = {"vox": vw.read_state(), "irr": rc.read_irradiance(), "counts": rc.read_counts(),
           "depth": rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(case.height, case.width),
           "normal": rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(case.height, case.width, 4),
           "probes": rc.read_buffer(_lib.GI_RC_PROBES).view(bind.PROBE_DTYPE),
           "rad": rc.read_atlas(_lib.GI_RC_RAD), "sh": rc.read_atlas(_lib.GI_RC_SH)}
    if case.shadow:
        res["shadow"] = rc.read_shadow()
    if debug:
        res["hits"] = rc.read_buffer(_lib.GI_RC_HITS).view(np.uint32).reshape(-1, 4)
        res["rad_traced"] = rc.read_atlas(_lib.GI_RC_RAD_TRACED)
    for h in (rc, vw, sg):
        h.destroy()
    return res


def oracle_scene(case):
    return gi_cases.posed(case.scene, *case.movers) if case.movers else case.scene


def run_oracle(case, depth, normal, shadow=None):
    v = case.vox
    st = bind.vox_build(oracle_scene(case), v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, case.scene.camera.eye)
    if shadow is not None:
        bind.vox_sun(st, case.frame, shadow)
    lay = dict(gi_cases.configs.cascade_layout(case.rc, case.width, case.height))
    out = bind.rc_solve(st, lay, case.frame, depth, normal, want_hit=True)
    return st, out


CASES = {"config0": gi_cases.config0, "room_lit": gi_cases.room_lit, "leak": gi_cases.leak,
         "leak_sun": gi_cases.leak_sun, "empty": gi_cases.empty, "single_triangle": gi_cases.single_triangle,
         "tiny": gi_cases.tiny,
         "room_lit_f32out": lambda: gi_cases.room_lit("f16-f32out"),
         "room_lit_irr16": lambda: gi_cases.room_lit("f32-irr16"),
         "overflow": gi_cases.overflow, "config1": gi_cases.config1,
         "batch_g4_l1": gi_cases.batch_g4_l1, "batch_g4_l4": gi_cases.batch_g4_l4,
         "batch_g32_l1": gi_cases.batch_g32_l1, "batch_g32_l4": gi_cases.batch_g32_l4,
         "movers_f16": gi_cases.movers_f16, "toon": gi_cases.toon, "toon_style_off": lambda: gi_cases.toon(False)}


@pytest.mark.parametrize("name", list(CASES))
def test_parity(ctx, name):
    case = CASES[name]()
    g = run_gpu(ctx, case)
    # G-buffer: the GPU raster against the oracle's, bit for bit
    depth, normal, _ = bind.raster_gbuffer(oracle_scene(case), case.frame, case.width, case.height)
    assert np.array_equal(g["depth"].view(np.uint32), depth.view(np.uint32)), "G-buffer depth differs"
    assert np.array_equal(g["normal"].astype(np.float32), normal), "G-buffer normal differs"
    shadow = None
    if case.shadow:   # the sun shadow map, bit for bit
        shadow = bind.shadow_render(oracle_scene(case), case.frame, case.shadow)
        assert np.array_equal(g["shadow"].view(np.uint32), shadow.view(np.uint32)), \
            f"shadow map differs at {(g['shadow'] != shadow).sum()} texels"
        assert (shadow < 1.0).any() or case.scene.triangle_count == 0
    st, o = run_oracle(case, depth, normal, shadow)
    # voxel world: every counter and every allocated word
    gv = g["vox"]
    assert np.array_equal(gv["hdr"], st["hdr"]), f"counters differ: {gv['hdr'][:32]} vs {st['hdr'][:32]}"
    nb = int(min(st["hdr"][0], case.vox.maxBricks))
    nv = int(min(st["hdr"][1], case.vox.maxVoxels))
    assert np.array_equal(gv["ptr"], st["ptr"]), "brick pointers differ"
    for k, n in (("occ", nb * 16), ("base", nb), ("code", nb), ("rep", nb * 512)):
        assert np.array_equal(gv[k][:n], st[k][:n]), f"{k} differs"
    assert np.array_equal(gv["attr"][:nv * 4], st["attr"][:nv * 4]), "voxel attributes differ"
    assert np.array_equal(gv["plane"][:nv].view(np.uint32), st["plane"][:nv].view(np.uint32)), "plane offsets differ"
    if case.shadow:
        assert np.array_equal(gv["sunvis"][:nv].view(np.uint32), st["sunvis"][:nv].view(np.uint32)), "sun visibility differs"
        sv = st["sunvis"][:nv]
        if case.name.startswith("leak") or case.name == "config1":
            assert (sv == 0.0).any() and (sv == 1.0).any(), "the case should hold shadowed and lit voxels"
    if case.name.startswith("toon"):   # the toon branch is reached: toon voxels (albedo alpha 255) are hit
        toon_vox = (gv["attr"][0:nv * 4:4] >> 24) == 255
        assert toon_vox.any() and not toon_vox.all()
        toon_hits = (g["hits"][:, 1] != 0xffffffff) & (g["hits"][:, 0] != 0xffffffff)
        assert toon_hits.any()
    if case.movers:
        objs, t = case.movers
        assert not np.array_equal(oracle_scene(case).positions, case.scene.positions)
    # probes and DDA hits
    assert np.array_equal(g["probes"].view(np.uint32), o["probes"].view(np.uint32)), "probes differ"
    assert np.array_equal(g["hits"], o["hit"]), f"DDA hits differ at {np.argwhere((g['hits'] != o['hit']).any(1))[:5].ravel()}"
    tol = _tol(case.rc.atlas)
    _close(g["rad_traced"], o["rad_traced"], tol, "traced radiance")
    _close(g["rad"], o["rad"], tol, "merged atlas")
    _close(g["sh"].reshape(-1)[: o["sh"].size], o["sh"].reshape(-1), tol, "SH")
    _close(g["irr"], o["irr"], tol, "irradiance")
    assert np.array_equal(g["counts"][:8], o["counts"][:8])


def test_bounce_parity(ctx):
    """Multi-bounce (bounce.ts) over three solves of the leak room with the sun's shadow map: the injected irradiance,
    the probe list and the irradiance of every solve bit-exact with the oracle's frames (the volume carries one frame
    of history, so the frames must agree in sequence)."""
    case = gi_cases.leak_sun(0.1, "f32", 512)
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    rc.set_frame(case.frame)
    rc.render_gbuffer(sg)
    rc.render_shadow(sg, case.shadow)
    vw.update(case.scene.camera.eye)
    rc.set_bounce(vw)
    depth, normal, _ = bind.raster_gbuffer(case.scene, case.frame, case.width, case.height)
    shadow = bind.shadow_render(case.scene, case.frame, case.shadow)
    v = case.vox
    st = bind.vox_build(case.scene, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, case.scene.camera.eye)
    bind.vox_sun(st, case.frame, shadow)
    ob = bind.Bounce(st)
    lay = dict(gi_cases.configs.cascade_layout(case.rc, case.width, case.height))
    nv = int(min(st["hdr"][1], v.maxVoxels))
    irr_prev = None
    try:
        for f in range(3):
            rc.solve(vw)
            g_irr = rc.read_irradiance()
            g_inj = rc.read_buffer(_lib.GI_RC_BOUNCE_INJ).view(np.float16).reshape(-1, 8)[:nv]
            g_list = rc.read_buffer(_lib.GI_RC_BOUNCE_LIST).view(np.uint32)
            inj = ob.frame(st, case.frame)[: nv * 6].reshape(nv, 6)
            assert g_list[1] == ob.list[1] and g_list[2] == ob.list[2] and g_list[0] == ob.list[0], \
                f"frame {f}: probe list {g_list[:3]} vs {ob.list[:3]}"
            assert np.array_equal(np.sort(g_list[4:4 + g_list[0]]), ob.list[4:4 + ob.list[0]]), f"frame {f}: listed probes differ"
            g6 = np.concatenate([g_inj[:, 0:3], g_inj[:, 4:7]], axis=1).astype(np.float32)
            assert np.array_equal(g6.view(np.uint32), inj.view(np.uint32)), \
                f"frame {f}: injected irradiance differs at {np.argwhere((g6 != inj).any(1))[:4].ravel()}"
            o = bind.rc_solve(st, lay, case.frame, depth, normal)
            _close(g_irr, o["irr"], 1e-4, f"irradiance, frame {f}")
            assert (inj > 0).any()
            if irr_prev is not None:
                assert not np.array_equal(g_irr, irr_prev)   # the second bounce arrives one frame later
            irr_prev = g_irr
    finally:
        for h in (rc, vw, sg):
            h.destroy()


def test_irr16_is_the_rounded_f32_solve(ctx):
    """irr16 stores the irradiance as rgba16float (the reference's rc.irr format): the same solve as the f32 one up
    to the store, which rounds to nearest even; the readback is half the bytes."""
    wide, narrow = gi_cases.room_lit("f32"), gi_cases.room_lit("f32-irr16")
    out = []
    for case in (wide, narrow):
        sg = gpu.SceneGpu(ctx, case.scene)
        vw = gpu.VoxWorld(sg, case.vox)
        rc = gpu.Rc(ctx, case.rc, case.width, case.height)
        rc.set_frame(case.frame)
        rc.render_gbuffer(sg)
        vw.update(case.scene.camera.eye)
        rc.solve(vw)
        raw = np.zeros(rc.irr_bytes(), np.uint8)
        rc.read_irradiance_raw(raw)
        out.append((raw, rc.read_atlas(_lib.GI_RC_RAD), rc.read_atlas(_lib.GI_RC_SH)))
        for h in (rc, vw, sg):
            h.destroy()
    (w_raw, w_rad, w_sh), (n_raw, n_rad, n_sh) = out
    assert n_raw.size * 2 == w_raw.size == wide.width * wide.height * 16
    assert np.array_equal(w_rad.view(np.uint32), n_rad.view(np.uint32)) and np.array_equal(w_sh.view(np.uint32), n_sh.view(np.uint32))
    w = w_raw.view(np.float32)
    assert (w > 0.0).any()
    assert np.array_equal(w.astype(np.float16).view(np.uint16), n_raw.view(np.uint16))


def test_walk_length_order_parity(ctx):
    """The config-1 solve traced in walk-length order (trace_order 2): three solves of one frame (the first in the
    order of the initial keys, the next in the order of the previous walks), then a frame with the camera moved (the
    keys of the previous frame's rays, which now walk elsewhere); the last solve of each frame checked bit for bit
    against the oracle — hits, traced and merged atlas, irradiance — and every ray traced once (the DDA counters of
    the atlas order)."""
    import dataclasses
    from rtgi import frame as fr, scenes as sc
    case = gi_cases.config1()
    cam = case.scene.camera
    cam2 = sc.Camera(tuple(a + b for a, b in zip(cam.eye, (0.12, 0.0, -0.08))),
                     tuple(a + b for a, b in zip(cam.target, (0.3, 0.0, 0.0))), cam.fov_y_deg, cam.near)
    F2 = gi_cases._frame(dataclasses.replace(case.scene, camera=cam2), case.width, case.height, case.rc,
                         sun_e=case.scene.sun_e, sky=case.scene.sky, shadow=True)
    # the same frame naming the first camera as the previous view
    F2p = fr.pack_frame(fr.FrameParams(cam=cam2, width=case.width, height=case.height, sun_dir=case.scene.sun_dir,
                                       sun_e=case.scene.sun_e, sky=case.scene.sky, cascades=case.rc.cascades,
                                       P=case.rc.P, s_min=case.rc.sMin, lift=case.rc.lift,
                                       light_view_proj=F2[64:80].tolist(), shadow_bias=(float(F2[157]), float(F2[158])),
                                       prev_cam=cam, prev_valid=True))
    assert np.array_equal(F2p[:32], F2[:32]) and int(F2p.view(np.uint32)[118]) == 1
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    got = []
    try:
        rc.set_frame(case.frame)
        rc.render_gbuffer(sg)
        rc.render_shadow(sg, case.shadow)
        vw.update(case.scene.camera.eye)
        rc.set_stats(1)
        rc.set_tuning(trace_order=0, trace_rays=1)
        rc.solve(vw)
        ref_counts = rc.read_counts()
        rc.set_tuning(trace_order=2, trace_rays=2)
        rc.set_debug_hits(True)
        for f, F in enumerate((case.frame, case.frame, case.frame, F2p)):
            if f == 3:
                rc.set_frame(F)
                rc.render_gbuffer(sg)
                vw.update(cam2.eye)
            rc.solve(vw)
            if f in (2, 3):
                got.append({"counts": rc.read_counts(),
                            "hits": rc.read_buffer(_lib.GI_RC_HITS).view(np.uint32).reshape(-1, 4),
                            "rad_traced": rc.read_atlas(_lib.GI_RC_RAD_TRACED), "rad": rc.read_atlas(_lib.GI_RC_RAD),
                            "irr": rc.read_irradiance(), "F": F, "eye": cam.eye if f == 2 else cam2.eye,
                            "depth": rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(case.height, case.width),
                            "normal": rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(case.height, case.width, 4)})
        shadow = rc.read_shadow()
    finally:
        for h in (rc, vw, sg):
            h.destroy()
    assert np.array_equal(got[0]["counts"], ref_counts), "DDA counters differ from the atlas order's"
    v = case.vox
    for g in got:
        st = bind.vox_build(case.scene, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, g["eye"])
        bind.vox_sun(st, g["F"], shadow)
        lay = dict(gi_cases.configs.cascade_layout(case.rc, case.width, case.height))
        o = bind.rc_solve(st, lay, g["F"], g["depth"], g["normal"].astype(np.float32), want_hit=True)
        assert np.array_equal(g["hits"], o["hit"]), "DDA hits differ"
        _close(g["rad_traced"], o["rad_traced"], 1e-4, "traced radiance")
        _close(g["rad"], o["rad"], 1e-4, "merged atlas")
        _close(g["irr"], o["irr"], 1e-4, "irradiance")
