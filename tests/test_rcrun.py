"""The runner entry (rtgi.rcrun, the reference's src/native/rc.ts for this path): host logic on the CPU, one short
run on the GPU."""
import json
import os

import numpy as np
import pytest

from rtgi import configs, rcrun


def test_stats_like_the_reference():
    s = rcrun.stats([4.0, 1.0, 3.0, 2.0, 5.0])
    assert s["median"] == 3.0 and s["mean"] == 3.0 and s["max"] == 5.0
    assert s["p05"] == pytest.approx(1.2) and s["p95"] == pytest.approx(4.8)


def test_pack_irradiance_tags_valid_pixels():
    irr = np.zeros((2, 3, 4), np.float32)
    irr[0, 1] = [1.0, 2.0, 3.0, 1.0]
    f = rcrun.pack_irradiance(irr)
    assert f.shape == (6, 4) and f.dtype == np.float32
    assert f[1].tolist() == [1.0, 2.0, 3.0, 1.0] and f[0, 3] == 0.0


def test_scene_names():
    s, v = rcrun.load_scene("room")
    assert s.triangle_count > 2000 and v["G"] == 8
    s2, _ = rcrun.load_scene("mix-3-obj5", pose_frame=12)
    s3, _ = rcrun.load_scene("mix-3")
    assert s2.triangle_count == s3.triangle_count + 5 * 12
    with pytest.raises(ValueError):
        rcrun.load_scene("sponza")
    with pytest.raises(ValueError):
        configs.vox_params({"v0": 0.1, "notAKey": 1})


@pytest.mark.gpu
def test_runner_writes_summaries(tmp_path):
    out = str(tmp_path)
    assert rcrun.main(["--scene", "room", "--configs", "screen-8-voxel-f32-dda64,screen-8-voxel-f16",
                       "--frames", "5", "--warmup", "2", "--width", "256", "--height", "256", "--out", out,
                       "--params", json.dumps({"cascades": 2}), "--dump-irr"]) == 0
    for name in ("screen-8-voxel-f32-dda64", "screen-8-voxel-f16"):
        s = json.load(open(os.path.join(out, f"{name}.summary.json")))
        assert s["config"] == name and s["resolution"] == "256x256"
        t = s["static"]["timing"]
        assert set(t) == {"vox", "giBuild", "giTrace", "giMerge", "giGather", "giTotal"}
        assert t["giTotal"]["median"] > 0 and len(s["tracer"]) == 2 and s["static"]["vox"]["bricks"] > 0
        irr = np.fromfile(os.path.join(out, f"{name}.static.irr.f32"), np.float32).reshape(-1, 4)
        assert irr.shape[0] == 256 * 256 and set(np.unique(irr[:, 3])) <= {0.0, 1.0}
    assert rcrun.main(["--scene", "room", "--vox-bench", "--out", out]) == 0
    vb = json.load(open(os.path.join(out, "vox-bench.default.json")))
    assert vb["total"]["median"] > 0 and vb["bricks"] > 0
