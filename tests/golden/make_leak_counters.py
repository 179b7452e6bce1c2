"""Extracts the voxel-build counters the reference recorded for its procedural leak rooms into leak_counters.json.

Run in the container that holds the reference checkout (it reads it; nothing at test time does):
    python tests/golden/make_leak_counters.py <reference checkout>
The source files are the reference's own measurement summaries (docs/reference/measurements/s2-voxel-stratabrick/
leak-<t>/world-32-voxel.summary.json): scene name and triangle count, voxParams, the static camera's readCounters()
(voxel.ts:908-918) and the camera that the leak scenes use (scenes.ts:276).
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_leak_counters.py <reference checkout>")
ref = sys.argv[1]
out = {}
for t in ("0.02", "0.05", "0.1", "0.2", "0.4"):
    p = os.path.join(ref, "docs/reference/measurements/s2-voxel-stratabrick", f"leak-{t}", "world-32-voxel.summary.json")
    d = json.load(open(p))
    v = d["static"]["vox"]
    out[t] = {"source": os.path.relpath(p, ref), "date": d["date"], "triangles": d["scene"]["triangles"],
              "voxParams": {k: d["voxParams"][k] for k in ("v0", "levels", "G", "maxBricks", "maxVoxels")},
              "bricks": v["bricks"], "voxels": v["voxels"], "brickOverflow": v["brickOverflow"],
              "bigOverflow": v["bigOverflow"], "voxelOverflow": v["voxelOverflow"],
              "bricksPerLevel": v["bricksPerLevel"], "bigPerLevel": v["bigPerLevel"]}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "leak_counters.json"), "w"), indent=1)
print("wrote", len(out), "scenes")
