"""gi_vox_build_noalloc: the voxel rebuild for callers that cannot allocate device memory.

A renderer that hands out every buffer from its own device pool, a thread in the middle of a CUDA-graph capture, or a
serving loop that must not stall the GPU with an allocation cannot let the library call cudaMalloc.  This entry point
takes the scene and the outputs in the caller's memory and uses a static device array for its scratch.  The GPU test
checks it against the allocating entry point (gi_vox_create + gi_vox_build) on two calls in a row: the outputs must
be bit-identical, the second call showing that the scratch left by the first does not leak into the result.  Before
them a call on a larger scene (the colonnade, which fills the brick pool) leaves the scratch full of another build's
representatives and lists.  This file is collected last so that a run stopping at the first failure has run every
other test already.
"""
import ctypes as C

import numpy as np
import pytest

import gi_cases
from rtgi import _lib, configs, gpu


def _params(v):
    return _lib.GiVoxParams(float(v.v0), v.levels, v.G, v.maxBricks, v.maxVoxels, v.dynBricks, 0)


def test_noalloc_rejects_sizes_past_its_scratch():
    lib = _lib.load()
    v = configs.vox_params({"v0": 0.1, "levels": 4, "G": 16, "maxBricks": 8192, "maxVoxels": 1 << 20})
    eye = (C.c_double * 3)(0.0, 0.0, 0.0)
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    st = lib.gi_vox_build_noalloc(C.byref(_params(v)), eye, dummy, dummy, 0, dummy, 0, dummy, 1,
                                  *([dummy] * 8), None)
    assert st == _lib.GI_ERR_INVALID
    assert b"max_bricks 8192 exceeds the static scratch" in lib.gi_last_error()


@pytest.mark.gpu
def test_noalloc_matches_allocating_build_twice():
    import torch
    case = gi_cases.room_lit()
    v = configs.vox_params({"v0": 0.08, "levels": 3, "G": 16, "maxBricks": 4096, "maxVoxels": 1 << 18})
    eye = case.scene.camera.eye
    # the allocating path
    ctx = gpu.Context(0)
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, v)
    vw.update(eye)
    vw.encode()
    ref = vw.read_state()
    for h in (vw, sg, ctx):
        h.destroy()
    # the caller's own device memory (allocated here by the test, not by the entry point)
    dev = torch.device("cuda", 0)
    s = case.scene
    pos4 = torch.zeros((s.positions.shape[0], 4), dtype=torch.float32, device=dev)
    nrm4 = torch.zeros_like(pos4)
    pos4[:, :3] = torch.from_numpy(s.positions).to(dev)
    nrm4[:, :3] = torch.from_numpy(s.normals).to(dev)
    tri = torch.from_numpy(s.tri.astype(np.uint32).view(np.int32)).to(dev).contiguous()
    mats = torch.from_numpy(s.material_array().view(np.uint8)).to(dev)
    nptr = v.levels * v.G ** 3
    out = {"hdr": torch.empty(64, dtype=torch.int32, device=dev), "ptr": torch.empty(nptr, dtype=torch.int32, device=dev),
           "occ": torch.empty(v.maxBricks * 16, dtype=torch.int32, device=dev),
           "base": torch.empty(v.maxBricks, dtype=torch.int32, device=dev),
           "code": torch.empty(v.maxBricks, dtype=torch.int32, device=dev),
           "attr": torch.empty(v.maxVoxels * 4, dtype=torch.int32, device=dev),
           "plane": torch.empty(v.maxVoxels, dtype=torch.float32, device=dev),
           "sunvis": torch.empty(v.maxVoxels, dtype=torch.float32, device=dev)}
    lib = _lib.load()
    e = (C.c_double * 3)(*[float(x) for x in eye])
    nb = int(min(ref["hdr"][0], v.maxBricks))
    nv = int(min(ref["hdr"][1], v.maxVoxels))
    assert nb > 100 and nv > 1000
    # a larger build first: the colonnade's 261k triangles fill the brick pool and the scratch
    from rtgi import scenes
    big = scenes.colonnade_scene(0)
    bpos = torch.zeros((big.positions.shape[0], 4), dtype=torch.float32, device=dev)
    bnrm = torch.zeros_like(bpos)
    bpos[:, :3] = torch.from_numpy(big.positions).to(dev)
    bnrm[:, :3] = torch.from_numpy(big.normals).to(dev)
    btri = torch.from_numpy(big.tri.astype(np.uint32).view(np.int32)).to(dev).contiguous()
    bmats = torch.from_numpy(big.material_array().view(np.uint8)).to(dev)
    be = (C.c_double * 3)(*[float(x) for x in big.camera.eye])
    st = lib.gi_vox_build_noalloc(C.byref(_params(v)), be, bpos.data_ptr(), bnrm.data_ptr(), bpos.shape[0],
                                  btri.data_ptr(), btri.shape[0], bmats.data_ptr(), len(big.materials),
                                  *[out[k].data_ptr() for k in ("hdr", "ptr", "occ", "base", "code", "attr", "plane", "sunvis")],
                                  None)
    assert st == 0, lib.gi_last_error()
    torch.cuda.synchronize()
    assert out["hdr"][0].item() > nb   # more bricks wanted than the room uses
    for call in range(2):
        for t in out.values():
            t.fill_(-1)   # garbage: every word the build owns must be rewritten
        torch.cuda.synchronize()
        st = lib.gi_vox_build_noalloc(C.byref(_params(v)), e, pos4.data_ptr(), nrm4.data_ptr(), pos4.shape[0],
                                      tri.data_ptr(), tri.shape[0], mats.data_ptr(), len(s.materials),
                                      *[out[k].data_ptr() for k in ("hdr", "ptr", "occ", "base", "code", "attr", "plane", "sunvis")],
                                      None)
        assert st == 0, lib.gi_last_error()
        torch.cuda.synchronize()
        got = {k: t.cpu().numpy().view(np.uint32) for k, t in out.items()}
        assert np.array_equal(got["hdr"], ref["hdr"]), f"call {call}: counters differ"
        assert np.array_equal(got["ptr"], ref["ptr"]), f"call {call}: brick pointers differ"
        for k, n in (("occ", nb * 16), ("base", nb), ("code", nb), ("attr", nv * 4)):
            assert np.array_equal(got[k][:n], ref[k][:n]), f"call {call}: {k} differs"
        for k in ("plane", "sunvis"):
            assert np.array_equal(got[k][:nv], ref[k][:nv].view(np.uint32)), f"call {call}: {k} differs"
