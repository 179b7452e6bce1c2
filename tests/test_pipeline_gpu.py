"""rtgi.pipeline: frames streamed with overlapped host copies give each frame the irradiance of a plain solve, with
the normals uploaded as rgba16f or as their three rgb halves (gi_rc_set_gbuffer_rgb16f)."""
import numpy as np
import pytest
import torch

import gi_cases
from rtgi import _lib, frame as fr, gpu, pipeline, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rgb", [False, True], ids=["rgba16f", "rgb16f"])
def test_pipeline_matches_plain_solves(rgb):
    case = gi_cases.room_lit()
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    vw.update(case.scene.camera.eye)
    cam_b = scenes.Camera(case.scene.camera.eye, (2.0, 1.0, 8.0), 60, 0.05)
    frames = [case.frame, gi_cases._frame(scenes.Scene(**{**case.scene.__dict__, "camera": cam_b}), case.width,
                                          case.height, case.rc, sun_e=fr.SUN_E, sky=fr.SKY)]
    inputs, expect = [], []
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    for F in frames:                       # the plain path: G-buffer, solve, readback, one frame at a time
        rc.set_frame(F)
        rc.render_gbuffer(sg)
        d = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).copy()
        n = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.uint16).copy()
        rc.solve(vw)
        out = np.zeros(rc.irr_bytes(), np.uint8)
        rc.read_irradiance_raw(out)
        expect.append(out)
        if rgb:
            n = np.ascontiguousarray(n.reshape(-1, 4)[:, :3]).reshape(-1)
        inputs.append((torch.from_numpy(F.copy()).pin_memory(), torch.from_numpy(d).pin_memory(),
                       torch.from_numpy(n).pin_memory()))
    rc.destroy()
    assert not np.array_equal(expect[0], expect[1])
    order = [0, 1, 1, 0, 1, 0, 0, 1]
    outs = [torch.empty(expect[0].size, dtype=torch.uint8).pin_memory() for _ in order]
    pipe = pipeline.FramePipeline(ctx, vw, case.rc, case.width, case.height, frames[0], inputs[0][1].data_ptr(),
                                  inputs[0][2].data_ptr(), slots=2, normal_rgb=rgb)
    for k, i in enumerate(order):
        f, d, n = inputs[i]
        pipe.submit(f.data_ptr(), d.data_ptr(), n.data_ptr(), outs[k].data_ptr())
    pipe.wait()
    for k, i in enumerate(order):
        assert np.array_equal(outs[k].numpy(), expect[i]), f"frame {k} (input {i}) differs from its plain solve"
    pipe.destroy()
    for h in (vw, sg, ctx):
        h.destroy()
