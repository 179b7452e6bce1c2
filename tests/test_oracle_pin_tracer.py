"""The oracle's world probes and DDA against the tracer statistics the reference recorded for its leak rooms.

The records (tests/golden/leak_tracer.json, made by tests/golden/make_leak_tracer.py) are ten runs of the reference
build of 2026-11-13: the five leak rooms, configs world-32-voxel and world-32-voxel-rc2 at 1920x1080 (P 32, caps sized
per room from a sizing pass, G-buffer relocation, voxel levels from voxScale 0.25, start offset 1 voxel, skip 0.5
voxel; clipmap 5 levels of G = 64 from 0.1 m).  What they pin here:

* the cascade layout: every recorded `intervals[c]` is `counts[c] * res_c^2` with res_c = 4 << min(c, resCap), and so is
  the oracle's (rays traced = live probes x directions, both resolution caps);
* the DDA step count (traceVox's loop iterations, brick skips and dropped-brick cells included, rc.ts:232-235): the
  mean steps per interval of every cascade agree with the record within 4 %, 1.2 % on average over the 50 values,
  and follow the record's changes with the wall thickness.

What they do not pin: the live probes per cascade.  The recorded c0 counts change with the wall thickness (9,572 to
10,530), while the room's inside, the only surface the static camera sees, is the same for every thickness (the walls
grow outwards; the voxel counters of the same runs, pinned in test_oracle_pin.py, confirm the geometry).  The current
registration (rc.ts:484-500: the 8 corners of each visible pixel's c0 cell) reads only that inside, so it gives one
count for all five rooms (12,157-12,169 here); the recorded ones came from a registration the reference no longer
has.  The test keeps that gap visible: the oracle's c0 count must be independent of the thickness.
"""
import json
import os

import numpy as np
import pytest

from oracle import bind
from rtgi import configs, frame as fr, scenes

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "leak_tracer.json")))
ROOMS = ("0.02", "0.05", "0.1", "0.2", "0.4")


def _solve(key):
    g = GOLD[key]
    t, cfg = key.split("/")
    s = scenes.leak_room(float(t))
    pr = g["params"]
    W, H = (int(x) for x in g["resolution"].split("x"))
    # the capacities only bound the tables: the reference sized them from the counts of a pass with its default
    # capacities (rcrun.ts:242-262); the default capacities, used here, hold every key
    p = configs.parse_config(cfg, {"cascades": pr["cascades"], "sMin": pr["sMin"], "lift": pr["lift"], "stats": 1})
    assert (p.P, p.resCap, p.voxScale, p.voxOffset, p.voxSkip, p.levelMap, p.relocate) == \
        (pr["P"], pr["resCap"], pr["voxScale"], pr["voxOffset"], pr["voxSkip"], pr["levelMap"], "gbuffer")
    lay = configs.world_layout(p)
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=g["sunDir"], sun_e=fr.SUN_E,
                                     sky=tuple(g["sky"]), cascades=p.cascades, P=p.P, s_min=p.sMin, lift=p.lift))
    depth, normal, _ = bind.raster_gbuffer(s, F, W, H)
    normal = normal.astype(np.float16).astype(np.float32)   # the G-buffer's rgba16float normals
    v = g["voxParams"]
    st = bind.vox_build(s, v["v0"], v["levels"], v["G"], v["maxBricks"], v["maxVoxels"], s.camera.eye,
                        coarse_from_triangles=True)
    o = bind.world_solve(st, lay, bind.WorldState(lay), F, depth, normal)
    return g, lay, o["counts"]


@pytest.fixture(scope="module")
def solved():
    return {k: _solve(k) for k in sorted(GOLD)}


def test_interval_layout(solved):
    for key, (g, lay, c) in solved.items():
        res = [4 << min(i, g["params"]["resCap"]) for i in range(5)]
        assert g["intervals"] == [n * r * r for n, r in zip(g["counts"], res)], key
        assert not c[8:13].any() and not c[16:21].any(), f"{key}: overflow or insert failure"
        assert [int(x) for x in c[24:29]] == [int(n) * r * r for n, r in zip(c[:5], res)], key
        assert not c[64:69].any() and g["atStepCap"] == [0] * 5, key


def test_mean_dda_steps_per_cascade(solved):
    rel = []
    for key, (g, lay, c) in solved.items():
        ours = [int(c[32 + i]) / int(c[24 + i]) for i in range(5)]
        for i, (a, b) in enumerate(zip(ours, g["meanSteps"])):
            assert abs(a / b - 1) < 0.04, f"{key} cascade {i}: {a:.4f} vs recorded {b}"
            rel.append(abs(a / b - 1))
    assert np.mean(rel) < 0.012, np.mean(rel)
    # the thick walls' voxels shorten cascade 3's walks in the record; the oracle shows the same
    thin, thick = (solved[f"{t}/world-32-voxel"] for t in ("0.1", "0.4"))
    m3 = lambda s: int(s[2][35]) / int(s[2][27])
    assert m3(thick) < m3(thin) and thick[0]["meanSteps"][3] < thin[0]["meanSteps"][3]


def test_c0_registration_is_blind_to_the_wall_thickness(solved):
    c0 = [int(solved[f"{t}/world-32-voxel"][2][0]) for t in ROOMS]
    rec = [solved[f"{t}/world-32-voxel"][0]["counts"][0] for t in ROOMS]
    assert (max(c0) - min(c0)) / min(c0) < 0.002, c0
    assert (max(rec) - min(rec)) / min(rec) > 0.09, rec
