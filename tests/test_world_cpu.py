"""The oracle's world probes (method 'world', rc.ts:248-570, 688-708, 775-927) against known answers and the
properties the CUDA path relies on: the ordered hash table is the one plain linear probing builds from the keys in
decreasing order, compact numbers the keys in slot order, parents are the grid points one cascade up, and the c0
history is a fixed point on a repeated frame."""
import math

import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import configs, frame as fr, scenes

NONE = 0xFFFFFFFF


def _hash32(x):
    h = x & 0xFFFFFFFF
    h ^= h >> 16; h = (h * 0x7FEB352D) & 0xFFFFFFFF
    h ^= h >> 15; h = (h * 0x846CA68B) & 0xFFFFFFFF
    h ^= h >> 16
    return h


def test_hash32_known_answers():
    for x in (0, 1, 2, 0x80000000, 0x9E3779B9, 0xFFFFFFFF, 123456789):
        assert bind.hash32(x) == _hash32(x)
    assert bind.hash32(0) == 0


def test_lod_for_is_floor_log2():
    F = np.zeros(160, np.float32)
    F[104:108] = [0.05, 0.001, 48, 0]
    k = 0.001 * 48 / 0.05
    for d in (0.01, 0.5, 1.0, 1.9, 2.5, 7.0, 33.0, 100.0, 500.0, 1e4, 1e9):
        y = max(float(np.float32(np.float32(np.float32(d) * np.float32(0.001)) * np.float32(48)) / np.float32(0.05)), 1.0)
        want = min(max(math.floor(math.log2(y)), 0), 14)
        assert bind.lod_for(F, d) == want, d
    # exactly at a power of two the exponent decides
    assert bind.lod_for(F, 8.0 / k) in (2, 3)


def _room_case(cfg="world-24-voxel-rc2-vrel-f32", caps=(8192, 4096, 2048, 1024, 512), W=160, H=120):
    s = scenes.room_scene(0)
    p = configs.parse_config(cfg, {"cascades": 5, "caps": list(caps) + [256] * 3})
    v = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    c = gi_cases.Case("room-world", s, W, H, v, p)
    c.frame = gi_cases._frame(s, W, H, p, sun_e=fr.SUN_E, sky=fr.SKY)
    return c


def _solve(case, state=None, frame=None):
    lay = configs.world_layout(case.rc)
    F = case.frame if frame is None else frame
    depth, normal, _ = bind.raster_gbuffer(case.scene, F, case.width, case.height)
    v = case.vox
    st = bind.vox_build(case.scene, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, case.scene.camera.eye)
    state = state or bind.WorldState(lay)
    return lay, state, bind.world_solve(st, lay, state, F, depth, normal.astype(np.float16).astype(np.float32))


@pytest.fixture(scope="module")
def solved():
    return _solve(_room_case())


def test_world_layout_matches_create_rc():
    p = configs.parse_config("world-48-voxel-rc2-vrel", {"cascades": 5})
    lay = configs.world_layout(p)
    caps = [1 << 18, 1 << 16, 1 << 14, 1 << 12, 1 << 11]
    assert [c["cap"] for c in lay["casc"]] == caps
    assert [c["res"] for c in lay["casc"]] == [4, 8, 16, 16, 16]          # rc2: res = 4 << min(i, 2)
    assert [c["hash_mask"] + 1 for c in lay["casc"]] == [2 * x for x in caps]   # nextPow2(2 cap)
    assert lay["relocate"] == 2 and lay["rays_total"] == sum(c * r * r for c, r in zip(caps, [4, 8, 16, 16, 16]))


def test_hash_tables_are_the_decreasing_order_tables(solved):
    lay, state, o = solved
    for c, L in enumerate(lay["casc"]):
        tab = o["keys"][L["hash_off"]:L["hash_off"] + L["hash_mask"] + 1]
        keys = np.sort(tab[tab != 0])[::-1]
        assert len(keys) == o["counts"][c] > 0
        ref = np.zeros_like(tab)
        mask = L["hash_mask"]
        for k in keys:   # plain linear probing, keys in decreasing order
            h = _hash32(int(k)) & mask
            while ref[h] != 0:
                h = (h + 1) & mask
            ref[h] = k
        assert np.array_equal(tab, ref)


def test_compact_numbers_keys_in_slot_order(solved):
    lay, state, o = solved
    for c, L in enumerate(lay["casc"]):
        sl = slice(L["hash_off"], L["hash_off"] + L["hash_mask"] + 1)
        occ = o["keys"][sl] != 0
        n = int(occ.sum())
        assert np.array_equal(o["slot_probe"][sl][occ], np.arange(n))
        # each probe carries its key's LOD, and s0 = sMin 2^lod
        pr = o["probes"][L["probe_off"]:L["probe_off"] + n]
        lod = (o["keys"][sl][occ] >> 27) & 15
        assert np.array_equal(pr["grid"][:, 3], lod.astype(np.int32))
        assert np.all(pr["pos"][:, 3] == np.float32(0.05) * np.exp2(lod.astype(np.float32)))


def test_parents_are_the_grid_points_above(solved):
    lay, state, o = solved
    for c in range(lay["cascades"] - 1):
        L, U = lay["casc"][c], lay["casc"][c + 1]
        n, nu = min(o["counts"][c], L["cap"]), min(o["counts"][c + 1], U["cap"])
        par = o["parents"][8 * L["probe_off"]:8 * (L["probe_off"] + n)].reshape(n, 8)
        g = o["probes"]["grid"][L["probe_off"]:L["probe_off"] + n]
        gu = o["probes"]["grid"][U["probe_off"]:U["probe_off"] + nu]
        linked = 0
        for i in range(n):
            for k in range(8):
                q = par[i, k]
                off = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
                if np.any((off > 0) & ((g[i, :3] & 1) == 0)):
                    assert q == NONE      # an even coordinate has one parent along that axis
                    continue
                if q == NONE:
                    continue              # absent, past the capacity, or hidden by voxels
                linked += 1
                assert np.array_equal(gu[q, :3], (g[i, :3] >> 1) + off) and gu[q, 3] == g[i, 3]
        assert linked > 0


def test_history_is_a_fixed_point_of_a_repeated_frame():
    case = _room_case()
    lay, state, o1 = _solve(case)
    assert state.hist_par == 1
    _, state, o2 = _solve(case, state)
    assert state.hist_par == 0
    assert np.array_equal(o1["irr"], o2["irr"]) and np.array_equal(o1["sh"], o2["sh"])
    # a moved camera keeps the probes it shares with the last frame half-way
    cam = case.scene.camera
    s3 = scenes.Scene(case.scene.name, case.scene.positions, case.scene.normals, case.scene.tri, case.scene.materials,
                      fr.Camera(tuple(np.add(cam.eye, (0.3, 0.0, 0.0))), tuple(np.add(cam.target, (0.3, 0.0, 0.0))),
                                cam.fov_y_deg, cam.near), case.scene.sun_dir)
    c3 = _room_case()
    c3.scene = s3
    c3.frame = gi_cases._frame(s3, c3.width, c3.height, c3.rc, sun_e=fr.SUN_E, sky=fr.SKY)
    _, fresh, o_fresh = _solve(c3)
    _, state, o3 = _solve(c3, state)
    assert not np.array_equal(o3["sh"], o_fresh["sh"])


def test_capacity_overflow_counts():
    case = _room_case(caps=(200, 100, 60, 40, 30))
    lay, state, o = _solve(case)
    assert o["counts"][8] == o["counts"][0] - 200 > 0
    n = lay["casc"][0]["cap"]
    assert (o["slot_probe"][:lay["casc"][0]["hash_mask"] + 1][o["keys"][:lay["casc"][0]["hash_mask"] + 1] != 0] == NONE).sum() \
        == o["counts"][8]
    assert n == 200


def test_colonnade_view_is_open():
    """The colonnade's camera stands in an aisle: its view reaches tens of metres (a camera inside a column sees the
    column's inside 0.3 m away)."""
    s = scenes.colonnade_scene(0)
    W, H = 160, 90
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H))
    depth, normal, tri = bind.raster_gbuffer(s, F, W, H)
    assert (depth > 0).mean() > 0.95
    assert len(np.unique(tri[tri != 0xFFFFFFFF])) > 200
    near = s.camera.near
    # reversed-Z infinite projection: view distance ~ near / depth
    assert np.median(near / depth[depth > 0]) > 2.0


# ---- worlds: instances, chunks and work items (world.ts) -------------------------------------------------------------

from rtgi import world as W

ROOM_V = {"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20}
INSTANCES = [(0, 0, 0), (12, 0, 0), (-14, 0, 3), (0, 0, 26)]


@pytest.fixture(scope="module")
def room_world():
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    s2, w = W.with_world(s, INSTANCES, float(v.v0), v.levels)
    return s, s2, w, v


def test_chunks_partition_the_rows(room_world):
    s, s2, w, v = room_world
    rows = np.sort(np.concatenate([ch.full for ch in w.chunks]))
    assert np.array_equal(rows, np.arange(s.triangle_count))
    P = np.asarray(s.positions, np.float64)
    for ch in w.chunks:
        tri = s.tri[ch.full]
        pts = P[tri[:, :3].reshape(-1)]
        assert np.all(pts.min(0) - W.MOTION_MARGIN >= np.array(ch.lo) - 1e-9)
        assert np.all(pts.max(0) + W.MOTION_MARGIN <= np.array(ch.hi) + 1e-9)
        c = P[tri[:, :3]].mean(1)        # every centroid in the chunk's 8 m cell
        assert len({tuple(np.floor(x / W.CHUNK).astype(int)) for x in c}) == 1
        assert ch.lod[0] is ch.full      # lod0Cell 0: level 0 voxelises the full triangles


def test_clustered_copies(room_world):
    s, s2, w, v = room_world
    T, V = s.triangle_count, s.positions.shape[0]
    assert w.rows == s2.tri.shape[0] == T + len(w.lod_table)
    assert s2.positions.shape[0] == V + w.lod_vertex_count
    assert (w.lod_table[:, :3] >= V).all() and (w.lod_table[:, :3] < V + w.lod_vertex_count).all()
    for ch in w.chunks:
        for L in range(1, v.levels):
            if len(ch.lod[L]):
                assert (ch.lod[L] >= T).all() and (ch.lod[L] < w.rows).all()
                # a clustered vertex lies in the cell of the vertices it replaces: within one cell of its triangle's
                cell = v.v0 * 2 ** (L - 1)
                src = s.tri[ch.full][:, :3].reshape(-1)
                lo = s.positions[src].min(0) - cell
                hi = s.positions[src].max(0) + cell
                pts = s2.positions[s2.tri[ch.lod[L]][:, :3].reshape(-1)]
                assert (pts >= lo - 1e-6).all() and (pts <= hi + 1e-6).all()


def test_items_start_at_the_finest_window(room_world):
    s, s2, w, v = room_world
    wins = W.windows(float(v.v0), v.levels, v.G, s.camera.eye)
    items = W.select_items(w, wins)
    assert {it.inst for it in items} == {0, 1, 2, 3} or {it.inst for it in items} >= {0, 1}
    for it in items:
        ch = next(c for c, ch in enumerate(w.chunks) if w.list_off[c][it.start] == it.list)
        o = w.instances[it.inst]
        box = (np.add(w.chunks[ch].lo, o), np.add(w.chunks[ch].hi, o))
        inside = [all(box[0][a] < wins[L][1][a] and box[1][a] > wins[L][0][a] for a in range(3)) for L in range(v.levels)]
        assert inside[it.start] and not any(inside[:it.start])
    rec, threads = W.item_records(items)
    assert threads == sum(it.count for it in items) and rec[0, 0] == 0


def test_single_instance_world_is_the_plain_build():
    s = scenes.room_scene(0)
    v = configs.vox_params(ROOM_V)
    s1, w1 = W.with_world(s, [(0, 0, 0)], float(v.v0), v.levels)
    eye = s.camera.eye
    a = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, eye)
    b = bind.vox_build(s1, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, eye, world=w1)
    assert all(it.start == 0 for it in W.select_items(w1, W.windows(float(v.v0), v.levels, v.G, eye)))
    for k in ("hdr", "ptr", "occ", "base", "code", "attr", "plane"):
        assert np.array_equal(a[k], b[k]), k


def test_instances_fill_the_coarse_levels(room_world):
    s, s2, w, v = room_world
    eye = s.camera.eye
    a = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, eye)
    b = bind.vox_build(s2, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, eye, world=w)
    assert b["hdr"][8] == a["hdr"][8]          # level 0 holds instance 0 only
    assert b["hdr"][9] > a["hdr"][9] and b["hdr"][10] > a["hdr"][10]


def test_world_requires_instance_zero_at_the_origin():
    with pytest.raises(ValueError):
        W.with_world(scenes.room_scene(0), [(1, 0, 0)], 0.08, 3)
