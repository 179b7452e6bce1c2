"""Parity of the dynamic layer (gi_dyn_*, dynlayer.ts) with the oracle, and of the traces that read it.

The lit room with 12 moving boxes as the scene's dynamic tail: the static rows go to the voxel rebuild
(gi_scene_set_static_count), the boxes are splatted into the dynamic layer, and the cascades read it in front of the
static hits (traceDyn).  Two frames with the boxes moved between them (the second empties the bricks only the first
wanted and flips the bitsets).  Compared word for word: the layer's header, pointers, bitsets, slot table, voxel masks
and data, then every DDA hit, traced and merged atlas entry and the irradiance, for screen and world probes."""
import dataclasses

import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, configs, frame as fr, gpu, movers, scenes

pytestmark = pytest.mark.gpu

VOX = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}
W, H, SHADOW = 256, 192, 512


def _scene():
    base = scenes.room_scene(0, n_boxes=60)
    s, objs = movers.with_moving_boxes(base, 12, scenes.PCG32(3, stream=5), area=(0.0, 0.0, 4.0, 4.0),
                                       height=(0.3, 1.5))
    return s, objs, base.triangle_count


def _posed(s, objs, t):
    P, N = s.positions.copy(), s.normals.copy()
    pos, nrm = objs.pose(t)
    P[objs.first:], N[objs.first:] = pos, nrm
    return dataclasses.replace(s, positions=P, normals=N)


def _eq(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    bad = a != b
    assert not bad.any(), f"{what}: {int(bad.sum())} of {bad.size} differ; first {np.argwhere(bad)[:3].ravel().tolist()}"


def _check_layer(g, dl, what):
    o = dl.arrays
    _eq(g["hdr"], o["hdr"], f"{what} header")
    _eq(g["ptr"], o["ptr"], f"{what} pointers")
    _eq(g["bits"], o["bits"], f"{what} bitsets")
    al = int(o["hdr"][8])
    _eq(g["meta"][:al], o["meta"][:al], f"{what} slots")
    _eq(g["mask"][:al * 16], o["mask"][:al * 16], f"{what} voxel masks")
    _eq(g["data"][:al * 512 * 13], o["data"][:al * 512 * 13], f"{what} voxel data")


@pytest.mark.parametrize("cfg", ["screen-8-voxel-f32-dda256", "world-24-voxel-rc2-vrel-f32"])
def test_dyn_layer_and_traces(cfg):
    s, objs, first = _scene()
    p = configs.parse_config(cfg, {"cascades": 4, "caps": [8192, 4096, 2048, 1024] + [256] * 4})
    v = configs.vox_params(VOX)
    world = cfg.startswith("world")
    lay = configs.world_layout(p) if world else configs.cascade_layout(p, W, H)
    F = gi_cases._frame(s, W, H, p, sun_e=fr.SUN_E, sky=fr.SKY, shadow=True)
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s)
    sg.set_static_count(first)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    dyn = gpu.DynLayer(vw, first, bricks=512)
    rc.set_dyn(dyn)
    rc.set_debug_hits(True)
    dl = st = state = None
    try:
        for f, t in enumerate((0.0, 0.6)):
            sc = _posed(s, objs, t)
            if f:
                sg.update_vertices(objs.first, sc.positions[objs.first:], sc.normals[objs.first:])
            rc.set_frame(F)
            rc.render_gbuffer(sg)
            rc.render_shadow(sg, SHADOW)
            vw.update(s.camera.eye)
            rc.solve(vw)
            g = dyn.read_state()
            depth = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H, W)
            normal = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H, W, 4).astype(np.float32)
            shadow = rc.read_shadow()
            # the oracle: the static rows voxelised, the moving boxes splatted
            _eq(shadow.view(np.uint32), bind.shadow_render(sc, F, SHADOW).view(np.uint32), f"frame {f} shadow map")
            st = bind.vox_build(dataclasses.replace(sc, tri=sc.tri[:first]), v.v0, v.levels, v.G, v.maxBricks,
                                v.maxVoxels, s.camera.eye)
            bind.vox_sun(st, F, shadow)
            if dl is None:
                dl = bind.Dyn(st, 512)
            dl.build(sc, st, first, sc.triangle_count, F, shadow)
            st["dyn"] = dl
            _check_layer(g, dl, f"frame {f}")
            assert g["hdr"][8] > 0 and g["hdr"][0] == g["hdr"][8], "bricks allocated, none dropped"
            assert ((g["data"][:int(g["hdr"][8]) * 512 * 13].reshape(-1, 13)[:, 6]) != 0).sum() > 100
            hits = rc.read_buffer(_lib.GI_RC_HITS).view(np.uint32).reshape(-1, 4)
            traced, irr = rc.read_atlas(_lib.GI_RC_RAD_TRACED), rc.read_irradiance()
            if world:
                if state is None:
                    state = bind.WorldState(lay)
                o = bind.world_solve(st, lay, state, F, depth, normal, want_hit=True)
                counts = rc.read_counts()
                _eq(counts, o["counts"], f"frame {f} counts")
                for c, L in enumerate(lay["casc"]):
                    n = min(int(o["counts"][c]), L["cap"])
                    rs = slice(L["rad_off"], L["rad_off"] + n * L["res"] ** 2)
                    _eq(hits[rs], o["hit"][rs], f"frame {f} cascade {c} hits")
            else:
                o = bind.rc_solve(st, lay, F, depth, normal, want_hit=True)
                _eq(hits, o["hit"], f"frame {f} hits")
                _eq(traced.view(np.uint32), o["rad_traced"].view(np.uint32), f"frame {f} traced atlas")
                # the layer is seen: some traced intervals are partly covered by a moving box
                T = o["rad_traced"][:, 3]
                assert ((T > 0.0) & (T < 1.0)).any()
            _eq(irr.view(np.uint32), o["irr"].view(np.uint32), f"frame {f} irradiance")
        assert dl.arrays["hdr"][10] == 2
    finally:
        for h in (rc, dyn, vw, sg, ctx):
            h.destroy()


BOUNCE = {"cell": 0.8, "dims": (16, 8, 16), "rays": 16, "div": 2}


def test_objects_receive_and_block_the_bounce():
    """The token obj (phase 31) over three frames with the boxes moving: before each frame's bounce volume the layer's
    voxels receive the previous volume (dynInject), and the volume's irradiance rays read the layer (bnTraceDyn).
    Compared with the oracle's frames: the layer's words after the injection (bit for bit), both bounce volumes, the
    probe list and the static voxels' injected irradiance (bit for bit), and the irradiance."""
    s, objs, first = _scene()
    p = configs.parse_config("screen-8-voxel-f32-dda256-obj", {"cascades": 4})
    assert p.objects
    v = configs.vox_params(VOX)
    lay = configs.cascade_layout(p, W, H)
    F = gi_cases._frame(s, W, H, p, sun_e=fr.SUN_E, sky=fr.SKY, shadow=True)
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, s)
    sg.set_static_count(first)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    dyn = gpu.DynLayer(vw, first, bricks=512, albedo=True)
    rc.set_dyn(dyn)
    rc.set_bounce(vw, **BOUNCE)
    dl = ob = None
    received = 0
    try:
        for f, t in enumerate((0.0, 0.3, 0.6)):
            sc = _posed(s, objs, t)
            if f:
                sg.update_vertices(objs.first, sc.positions[objs.first:], sc.normals[objs.first:])
            rc.set_frame(F)
            rc.render_gbuffer(sg)
            rc.render_shadow(sg, SHADOW)
            vw.update(s.camera.eye)
            rc.solve(vw)
            g = dyn.read_state()
            g_vol = rc.read_buffer(_lib.GI_RC_BOUNCE_VOL).view(np.float16).astype(np.float32).reshape(2, -1)
            g_list = rc.read_buffer(_lib.GI_RC_BOUNCE_LIST).view(np.uint32)
            depth = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H, W)
            normal = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H, W, 4).astype(np.float32)
            shadow = rc.read_shadow()
            irr = rc.read_irradiance()
            st = bind.vox_build(dataclasses.replace(sc, tri=sc.tri[:first]), v.v0, v.levels, v.G, v.maxBricks,
                                v.maxVoxels, s.camera.eye)
            bind.vox_sun(st, F, shadow)
            if dl is None:
                dl = bind.Dyn(st, 512, albedo=True)
                ob = bind.Bounce(st, objects=True, **BOUNCE)
            dl.build(sc, st, first, sc.triangle_count, F, shadow)
            st["dyn"] = dl
            before = dl.arrays["data"].copy()
            inj = ob.frame(st, F)
            received += int((dl.arrays["data"] != before).sum())
            _check_layer(g, dl, f"frame {f} (after dynInject)")
            for k in range(2):
                _eq(g_vol[k].view(np.uint32), ob.vol[k].view(np.uint32), f"frame {f} bounce volume {k}")
            _eq(g_list[:3], ob.list[:3], f"frame {f} probe list header")
            nv = int(min(st["hdr"][1], v.maxVoxels))
            g_inj = rc.read_buffer(_lib.GI_RC_BOUNCE_INJ).view(np.float16).reshape(-1, 8)[:nv]
            g6 = np.concatenate([g_inj[:, 0:3], g_inj[:, 4:7]], axis=1).astype(np.float32)
            _eq(g6.view(np.uint32), inj[: nv * 6].reshape(nv, 6).view(np.uint32), f"frame {f} injected irradiance")
            o = bind.rc_solve(st, lay, F, depth, normal)
            valid = o["irr"][..., 3] > 0
            np.testing.assert_allclose(irr[valid], o["irr"][valid], rtol=1e-4, atol=1e-4 * np.abs(o["irr"]).max(),
                                       err_msg=f"frame {f} irradiance")
        assert received > 100, "the moving boxes received the volume's light"
        # a graph captured with the objects on is refused once they are turned off
        import torch
        st = torch.cuda.Stream()
        torch.cuda.synchronize()
        rc.graph_capture(vw, st)
        rc.graph_launch(st)
        rc.set_objects(False)
        with pytest.raises(_lib.GiError):
            rc.graph_launch(st)
        st.synchronize()
    finally:
        for h in (rc, dyn, vw, sg, ctx):
            h.destroy()
