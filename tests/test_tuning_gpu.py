"""Launch tuning (gi_rc_tuning / gi_vox_tuning) never changes a result, and the autotuner picks valid settings."""
import numpy as np
import pytest

import gi_cases
from rtgi import _lib, autotune, gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.destroy()


def _solve(ctx, case, rc_tuning=None, vox_tuning=None):
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    try:
        if rc_tuning:
            rc.set_tuning(**rc_tuning)
        if vox_tuning:
            vw.set_tuning(**vox_tuning)
        rc.set_frame(case.frame)
        rc.render_gbuffer(sg)
        vw.update(case.scene.camera.eye)
        rc.set_debug_hits(True)
        rc.solve(vw)
        rc.solve(vw)   # the walk-length order (trace_order 2) uses the first solve's walks in the second
        st = vw.read_state()
        out = {"irr": rc.read_buffer(_lib.GI_RC_RAD), "sh": rc.read_buffer(_lib.GI_RC_SH),
               "hits": rc.read_buffer(_lib.GI_RC_HITS), "traced": rc.read_buffer(_lib.GI_RC_RAD_TRACED)}
        irr = np.zeros(rc.irr_bytes(), np.uint8)
        rc.read_irradiance_raw(irr)
        out["irr_out"] = irr
        for k in ("hdr", "ptr", "occ", "base", "code", "attr", "plane"):
            out["vox_" + k] = st[k]
    finally:
        for h in (rc, vw, sg):
            h.destroy()
    return out


VARIANTS = [
    ({"trace_order": 1}, None),
    ({"trace_order": 2}, None),
    ({"trace_order": 2, "trace_rays": 2, "trace_blocks": 4}, None),
    ({"trace_rays": 4, "trace_blocks": 2}, None),
    ({"trace_order": 1, "trace_rays": 2, "trace_blocks": 16}, None),
    ({"gather_shape": 0}, None),
    ({"gather_shape": 1, "merge_threads": 64}, None),
    ({"gather_shape": 2, "merge_threads": 512}, None),
    (None, {"chunk_cells": 32, "blocks": 2}),
    (None, {"chunk_cells": 1024, "blocks": 16}),
]


@pytest.mark.parametrize("name", ["room_lit", "leak"])
def test_tuning_does_not_change_results(ctx, name):
    case = {"room_lit": gi_cases.room_lit, "leak": gi_cases.leak}[name]()
    ref = _solve(ctx, case)
    assert ref["irr_out"].any()
    for rt, vt in VARIANTS:
        got = _solve(ctx, case, rt, vt)
        for k in ref:
            assert np.array_equal(got[k], ref[k]), f"{k} differs under rc {rt} vox {vt}"


def test_tuning_rejects_bad_values(ctx):
    case = gi_cases.config0()
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    try:
        for bad in ({"trace_rays": 3}, {"trace_order": 3}, {"trace_blocks": 0}, {"gather_shape": 4},
                    {"merge_threads": 100}):
            with pytest.raises(_lib.GiError):
                rc.set_tuning(**bad)
        assert rc.get_tuning() == {"trace_order": 0, "trace_rays": 1, "trace_blocks": 8, "gather_shape": 3,
                                   "merge_threads": 256}
    finally:
        rc.destroy()


def test_autotuner_picks_and_caches(ctx, tmp_path):
    case = gi_cases.room_lit()
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    try:
        rc.set_frame(case.frame)
        rc.render_gbuffer(sg)
        vw.update(case.scene.camera.eye)
        path = str(tmp_path / "tune.json")
        tu = autotune.Autotuner(path, reps=3)
        res = tu.tune(rc, vw)
        assert set(res["ms"]) == {"giTrace", "giMerge", "giGather", "vox"}
        assert rc.get_tuning() == res["rc"] and vw.get_tuning() == res["vox"]
        again = autotune.Autotuner(path).tune(rc, vw)     # from the file, no timing
        assert again["rc"] == res["rc"] and again["vox"] == res["vox"]
    finally:
        for h in (rc, vw, sg):
            h.destroy()
