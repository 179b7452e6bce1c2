"""Batches of uneven solves (one CUDA graph of parallel solve chains) give, solve by solve, exactly what each solve
gives alone; and the batch spec generator follows the batch configuration's distributions."""
import math

import numpy as np
import pytest

from rtgi import batch, scenes


def small_specs(n=5):
    specs = []
    for s in range(n):
        sp = scenes.batch_spec(100 + s)
        sp["tris"] = min(sp["tris"], 30_000)
        sp["width"], sp["height"] = min(sp["width"], 480), min(sp["height"], 270)
        specs.append(sp)
    return specs


def test_batch_spec_ranges():
    specs = [scenes.batch_spec(s) for s in range(64)]
    assert all(5_000 <= s["tris"] <= 500_000 for s in specs)
    assert {s["G"] for s in specs} == {4, 8, 16, 32}            # 32^3 .. 256^3 voxels per level
    assert {s["levels"] for s in specs} == {1, 2, 3, 4}
    assert {s["cascades"] for s in specs} == {2, 3, 4, 5}
    assert all(320 <= s["width"] <= 1920 and 180 <= s["height"] <= 1080 for s in specs)
    logs = [math.log(s["tris"]) for s in specs]
    assert abs(np.mean(logs) - (math.log(5e3) + math.log(5e5)) / 2) < 0.6   # log-uniform
    sc = scenes.mixed_scene(3, 20_000)
    assert 18_000 <= sc.triangle_count <= 21_000


@pytest.mark.gpu
def test_batch_equals_solves_alone():
    import torch
    from rtgi import gpu
    ctx = gpu.Context(0)
    stream = torch.cuda.Stream()
    solves = [batch.make_solve(ctx, sp, stream=stream) for sp in small_specs()]
    alone = []
    for x in solves:
        x.rc.solve(x.vox, stream)
        alone.append(x.rc.read_irradiance(stream).copy())
        x.rc.graph_capture(x.vox, stream)
    b = batch.make_batch(ctx, solves, stream)
    for rep in range(2):
        b.launch(stream)
        stream.synchronize()
        for i, x in enumerate(solves):
            got = x.rc.read_irradiance(stream)
            assert np.array_equal(got.view(np.uint32), alone[i].view(np.uint32)), f"solve {i} differs in the batch (launch {rep})"
    # a solve replayed alone after the batch still gives its own result
    solves[2].rc.graph_launch(stream)
    assert np.array_equal(solves[2].rc.read_irradiance(stream).view(np.uint32), alone[2].view(np.uint32))
    # the same batch pass by pass: one launch per cascade pass over every solve
    b.capture_passes(stream)
    for x in solves:   # first overwrite every output with a solve under twice the sun
        f2 = np.array(x.frame, np.float32).copy()
        f2[92:95] *= 2.0
        x.rc.set_frame(f2, stream)
        x.rc.solve(x.vox, stream)
        assert not np.array_equal(x.rc.read_irradiance(stream), alone[solves.index(x)])
        x.rc.set_frame(x.frame, stream)
    for rep in range(2):
        b.launch(stream)
        stream.synchronize()
        for i, x in enumerate(solves):
            got = x.rc.read_irradiance(stream)
            assert np.array_equal(got.view(np.uint32), alone[i].view(np.uint32)), f"solve {i} differs pass by pass (launch {rep})"
    # and every solve of the batch against the oracle, on the oracle's own G-buffer (the batched pass kernels:
    # k_setup_batch, k_trace_batch, k_merge_batch, k_gather_batch)
    from oracle import bind
    from rtgi import configs
    for i, x in enumerate(solves):
        W, H = x.spec["width"], x.spec["height"]
        p, v = batch.solve_params(x.spec)
        depth, normal, _ = bind.raster_gbuffer(x.scene, x.frame, W, H)
        st = bind.vox_build(x.scene, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, x.scene.camera.eye)
        o = bind.rc_solve(st, configs.cascade_layout(p, W, H), x.frame, depth, normal)
        got = x.rc.read_irradiance(stream)
        assert np.array_equal(got.view(np.uint32), o["irr"].view(np.uint32)), f"solve {i} differs from the oracle"
    b.destroy()
    for x in solves:
        x.destroy()
    ctx.destroy()
