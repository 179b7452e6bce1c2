"""Autotuner of the launch shapes of one solve (no counterpart in the reference, whose workgroup sizes are fixed in its
WGSL).  The tunables change how work is laid onto the GPU, never the result (tested bit-exact):

  giTrace   trace_order (probe-major: a warp's lanes take an 8 x 4 tile of a probe's directions, alike walks;
            direction-major: one direction over 32 neighbouring probes, coherent voxel paths), trace_rays (rays per
            lane per queue fetch), trace_blocks (resident blocks per SM of the persistent trace).  The walk-length
            order (trace_order 2) is left out: it pays only while the camera holds still, and the tuner's repeated
            solves of one frame would favour it for any workload.
  giMerge   merge_threads (block size)
  giGather  gather_shape (16x16, 32x8 or 8x32 pixels per block, or warps on probe-aligned tiles)
  vox       chunk_cells (cells per big-triangle work item of voxBits), blocks (resident blocks per SM)

Each pass's tunables only move that pass's time, so the search is per pass: every combination of one pass's
tunables, the others held, timed by the solve's per-pass CUDA events (median of `reps` solves).  Results are cached
per solve shape (resolution, cascades, atlas, clipmap, triangle count to a power of two), optionally in a JSON file.
"""
from __future__ import annotations

import itertools
import json
import os
import statistics
from typing import Dict, Optional

RC_GROUPS = {
    "giTrace": {"trace_order": [0, 1], "trace_rays": [1, 2, 4], "trace_blocks": [4, 8, 16]},
    "giMerge": {"merge_threads": [128, 256, 512]},
    "giGather": {"gather_shape": [0, 1, 2, 3]},
}
VOX_GROUPS = {"vox": {"chunk_cells": [32, 64, 128, 256, 512], "blocks": [4, 8, 16]}}


def shape_key(rc, vox) -> str:
    p, v = rc.params, vox.params
    ntris = int(vox.scene.scene.triangle_count) if getattr(vox.scene, "scene", None) is not None else 0
    return (f"{rc.width}x{rc.height}-c{p.cascades}-P{p.P}-{p.atlas}-L{v.levels}-G{v.G}-"
            f"t{max(0, ntris - 1).bit_length()}")


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, reps: int = 5):
        self.cache_path = cache_path
        self.reps = reps
        self.cache: Dict[str, dict] = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def _time(self, rc, vox, stream, pass_name: str) -> float:
        ms = []
        for _ in range(self.reps):
            rc.solve(vox, stream)
            ms.append(rc.pass_times()[pass_name])
        return statistics.median(ms)

    def tune(self, rc, vox, stream=None) -> dict:
        """Picks and applies the launch shapes for this (rc, vox); returns {"rc": {...}, "vox": {...}, "ms": {...}}.
        Needs the frame, G-buffer and voxel window set (it runs solves)."""
        key = shape_key(rc, vox)
        hit = self.cache.get(key)
        if hit is not None:
            rc.set_tuning(**hit["rc"])
            vox.set_tuning(**hit["vox"])
            return hit
        was_timing = False
        rc.set_timing(True)
        try:
            rc.solve(vox, stream)                      # warm
            best_ms = {}
            for pass_name, space in list(RC_GROUPS.items()) + list(VOX_GROUPS.items()):
                target = vox if pass_name == "vox" else rc
                names = list(space)
                best = None
                for combo in itertools.product(*[space[n] for n in names]):
                    target.set_tuning(**dict(zip(names, combo)))
                    t = self._time(rc, vox, stream, pass_name)
                    if best is None or t < best[0]:
                        best = (t, dict(zip(names, combo)))
                target.set_tuning(**best[1])
                best_ms[pass_name] = best[0]
        finally:
            rc.set_timing(was_timing)
        res = {"rc": rc.get_tuning(), "vox": vox.get_tuning(), "ms": best_ms}
        self.cache[key] = res
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
        return res
