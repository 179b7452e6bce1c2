"""A bounded device wait that runs out is reported to the caller, and the context stays usable.

The rebuild's chained scans wait on the parts before them with a bounded spin (csrc/gi_scan.cuh); a part that gives
up sets header word 6.  gi_vox_debug_hold_scan makes one part of the brick-allocation scan publish nothing, so the
next part's wait must run out: the kernels return, the stream completes, gi_vox_read_counters returns GI_ERR_TIMEOUT
with a message (the reference reports its build's failures as counters the host reads, voxel.ts:463,586), and the
next rebuild without the hold is correct again.  No GPU fault is involved: the wait simply gives up."""
import time

import numpy as np
import pytest

from oracle import bind
from rtgi import _lib, configs, gpu, scenes

pytestmark = pytest.mark.gpu


def test_scan_wait_runs_out_and_is_reported():
    ctx = gpu.Context(0)
    s = scenes.room_scene(0)
    vp = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    sg = gpu.SceneGpu(ctx, s)
    vw = gpu.VoxWorld(sg, vp)
    try:
        vw.update(s.camera.eye)
        vw.encode()
        good = vw.read_counters()["hdr"].copy()
        assert good[6] == 0
        vw.debug_hold_scan(0)            # part 0 of the brick scan never publishes: part 1 waits and gives up
        t0 = time.perf_counter()
        vw.encode()
        with pytest.raises(_lib.GiError) as e:
            vw.read_counters()
        waited = time.perf_counter() - t0
        assert e.value.status == _lib.GI_ERR_TIMEOUT and "gave up" in str(e.value)
        assert waited < 10.0, waited
        vw.debug_hold_scan(-1)
        vw.encode()
        again = vw.read_counters()["hdr"]
        assert np.array_equal(again, good)
        st = bind.vox_build(s, vp.v0, vp.levels, vp.G, vp.maxBricks, vp.maxVoxels, s.camera.eye)
        assert np.array_equal(again, st["hdr"])
    finally:
        for h in (vw, sg, ctx):
            h.destroy()
