"""Extracts the world-probe and tracer statistics the reference recorded for its procedural leak rooms into
leak_tracer.json.

Run in the container that holds the reference checkout (it reads it; nothing at test time does):
    python tests/golden/make_leak_tracer.py <reference checkout>
Sources: docs/reference/measurements/s2-voxel-stratabrick/leak-<t>/world-32-voxel{,-rc2}.summary.json, written by
the reference's runner (rcrun.ts runConfig): the run parameters (`params`, `voxParams`, resolution), the live probes
per cascade of the static camera (`static.counts`, Rc.readCounts words 0-4) and the tracer statistics of one more
static frame with stats on (`tracer[c]`: intervals = rays traced, meanSteps = DDA steps / intervals to 4 decimals,
rcrun.ts traceStats).
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_leak_tracer.py <reference checkout>")
ref = sys.argv[1]
out = {}
for t in ("0.02", "0.05", "0.1", "0.2", "0.4"):
    for cfg in ("world-32-voxel", "world-32-voxel-rc2"):
        p = os.path.join(ref, "docs/reference/measurements/s2-voxel-stratabrick", f"leak-{t}", f"{cfg}.summary.json")
        d = json.load(open(p))
        out[f"{t}/{cfg}"] = {
            "source": os.path.relpath(p, ref), "date": d["date"], "resolution": d["resolution"],
            "params": {k: d["params"][k] for k in ("method", "P", "cascades", "sMin", "kInterval", "regStride", "lift",
                                                  "caps", "world", "levelMap", "voxScale", "voxOffset", "voxSkip",
                                                  "resCap", "relocate")},
            "voxParams": d["voxParams"], "sky": d["sky"], "sunDir": d["scene"]["sunDir"],
            "counts": d["static"]["counts"], "overflow": d["static"]["overflow"],
            "intervals": [c["intervals"] for c in d["tracer"]], "meanSteps": [c["meanSteps"] for c in d["tracer"]],
            "atStepCap": [c["atStepCap"] for c in d["tracer"]]}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "leak_tracer.json"), "w"), indent=1)
print("wrote", len(out), "runs")
