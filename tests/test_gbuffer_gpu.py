"""The binned G-buffer raster against the oracle's brute-force raster (every pixel of every triangle's screen box),
bit for bit, on dense scenes with moving boxes and with the per-tile lists forced to overflow."""
import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, frame as fr, gpu, scenes, serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.destroy()


def _render(ctx, scene, frame, W, H, p, capacity=None, poses=()):
    sg = gpu.SceneGpu(ctx, scene)
    rc = gpu.Rc(ctx, p, W, H)
    out = []
    try:
        if capacity is not None:
            sg.set_raster_capacity(capacity)
        rc.set_frame(frame)
        for pose in poses or [None]:
            if pose is not None:
                sg.update_vertices(*pose)
            rc.render_gbuffer(sg)
            out.append((rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(H, W),
                        rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(H, W, 4)))
    finally:
        rc.destroy()
        sg.destroy()
    return out


def _check(scene, frame, W, H, got):
    depth, normal, _ = bind.raster_gbuffer(scene, frame, W, H)
    assert np.array_equal(got[0].view(np.uint32), depth.view(np.uint32)), \
        f"depth differs at {np.argwhere(got[0].view(np.uint32) != depth.view(np.uint32))[:4].tolist()}"
    assert np.array_equal(got[1].astype(np.float32), normal), "normal differs"
    assert (depth > 0).any()


@pytest.mark.parametrize("seed", [1, 3])
def test_moving_box_scenes(ctx, seed):
    spec = scenes.batch_spec(seed)
    s, objs = serve.serving_scene(spec, 40)
    p = serve.configs.parse_config("screen-8-voxel-f16-dda256", {"cascades": spec["cascades"]})
    W, H = spec["width"], spec["height"]
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=s.sun_e, sky=s.sky,
                                     cascades=p.cascades, P=p.P))
    pos, nrm = objs.pose(0.75)
    got = _render(ctx, s, F, W, H, p, poses=[(objs.first, pos, nrm)])
    moved = scenes.Scene(**{**s.__dict__})
    moved.positions = s.positions.copy()
    moved.normals = s.normals.copy()
    moved.positions[objs.first:] = pos
    moved.normals[objs.first:] = nrm
    _check(moved, F, W, H, got[0])


def test_list_overflow_gives_the_same_gbuffer(ctx):
    case = gi_cases.room_lit("f32")
    full = _render(ctx, case.scene, case.frame, case.width, case.height, case.rc)[0]
    tiny = _render(ctx, case.scene, case.frame, case.width, case.height, case.rc, capacity=300)[0]
    assert np.array_equal(full[0].view(np.uint32), tiny[0].view(np.uint32))
    assert np.array_equal(full[1].view(np.uint16), tiny[1].view(np.uint16))
    _check(case.scene, case.frame, case.width, case.height, tiny)
