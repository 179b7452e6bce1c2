"""The oracle's voxel build against the counters the reference recorded for its procedural leak rooms.

The records (tests/golden/leak_counters.json, made by tests/golden/make_leak_counters.py from the reference's
measurement summaries) come from the reference build of 2026-11-13, which voxelised every level from the triangles;
the oracle reproduces that build with coarse_from_triangles=1 and must match every counter, the big-triangle lists
per level included.  The current build (coarse levels reduced from the finer one, voxel.ts:16-19) must give the
same bricks and voxels: every coarse voxel of these scenes is the OR of its children.
"""
import json
import os

import pytest

from oracle import bind
from rtgi import scenes

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "leak_counters.json")))


@pytest.mark.parametrize("t", sorted(GOLD))
@pytest.mark.parametrize("coarse_from_triangles", [True, False])
def test_leak_room_counters(t, coarse_from_triangles):
    g = GOLD[t]
    s = scenes.leak_room(float(t))
    assert s.triangle_count == g["triangles"]
    vp = g["voxParams"]
    st = bind.vox_build(s, vp["v0"], vp["levels"], vp["G"], vp["maxBricks"], vp["maxVoxels"], s.camera.eye,
                        coarse_from_triangles=coarse_from_triangles)
    h = [int(x) for x in st["hdr"]]
    NL = vp["levels"]
    assert min(h[0], vp["maxBricks"]) == g["bricks"]
    assert h[1] == g["voxels"]
    assert (h[2], h[3], h[4]) == (g["brickOverflow"], g["bigOverflow"], g["voxelOverflow"])
    assert h[8:8 + NL] == g["bricksPerLevel"]
    if coarse_from_triangles:
        assert h[16:16 + NL] == g["bigPerLevel"]
    else:
        assert h[16] == g["bigPerLevel"][0] and h[17:16 + NL] == [0] * (NL - 1)
