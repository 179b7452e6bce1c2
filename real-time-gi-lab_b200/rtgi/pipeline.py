"""Frames streamed through the drop-in path with the host copies overlapped (no counterpart in the reference, which
submits one frame per queue and maps its readback buffer when the frame is done, rcrun.ts:322-335).

Each frame's inputs (the 640-byte frame block, depth f32, normal rgba16f or its rgb halves) are copied from pinned host memory on an
upload stream, the frame is solved (voxel rebuild + cascades, one captured graph) on the compute stream, and its
irradiance is copied back on a download stream.  `slots` cascade sets take turns (two by default; three measured the
same on the colonnade), so the upload of the next frame and the download of the last run while frame k is solved: the step time approaches the slower of the PCIe copies and the solve
instead of their sum.  The voxel world is shared and only the compute stream touches it, so solves stay in order.
"""
from __future__ import annotations

from typing import List

from . import gpu


class FramePipeline:
    def __init__(self, ctx: gpu.Context, vox: gpu.VoxWorld, params, width: int, height: int, frame, depth_ptr: int,
                 normal_f16_ptr: int, slots: int = 2, shadow=None, tuning=None, normal_rgb: bool = False):
        """frame/depth/normal: a first frame's inputs (frame as an array, the G-buffer as pinned host pointers), used
        to capture each slot's graph.  shadow: (SceneGpu, size) to give every slot the sun's shadow map drawn from
        that frame (a static sun and scene; draw it again with Rc.render_shadow when they move).  tuning: launch
        shapes for every slot (Rc.set_tuning's keywords; results do not depend on them).  normal_rgb: the host
        normals are three halves per pixel (6 bytes over the bus instead of 8; the path reads no alpha)."""
        import torch
        self.torch = torch
        self.vox = vox
        self.rgb = normal_rgb
        self.up, self.comp, self.down = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        self.rcs: List[gpu.Rc] = []
        for _ in range(slots):
            rc = gpu.Rc(ctx, params, width, height)
            rc.set_frame(frame, self.comp)
            rc.set_gbuffer_ptrs(depth_ptr, normal_f16_ptr, self.comp, rgb=normal_rgb)
            if tuning:
                rc.set_tuning(**tuning)
            if shadow is not None:
                rc.render_shadow(shadow[0], shadow[1], self.comp)
            rc.graph_capture(vox, self.comp)
            self.rcs.append(rc)
        self.uploaded = [torch.cuda.Event() for _ in range(slots)]
        self.solved = [torch.cuda.Event() for _ in range(slots)]
        self.downloaded = [torch.cuda.Event() for _ in range(slots)]
        for i in range(slots):
            self.uploaded[i].record(self.up)
            self.solved[i].record(self.comp)
            self.downloaded[i].record(self.down)
        self.k = 0
        self.comp.synchronize()

    @property
    def irr_bytes(self) -> int:
        return self.rcs[0].irr_bytes()

    def submit(self, frame_ptr: int, depth_ptr: int, normal_f16_ptr: int, out_ptr: int) -> int:
        """Queues one frame: inputs from pinned host memory, irradiance (as stored) into pinned host memory at out_ptr.
        Returns the slot; the output is complete once done(slot) (or wait()) says so."""
        s = self.k % len(self.rcs)
        rc = self.rcs[s]
        self.up.wait_event(self.solved[s])          # the slot's previous solve has read its inputs
        rc.set_frame_ptr(frame_ptr, self.up)
        rc.set_gbuffer_ptrs(depth_ptr, normal_f16_ptr, self.up, rgb=self.rgb)
        self.uploaded[s].record(self.up)
        self.comp.wait_event(self.uploaded[s])
        self.comp.wait_event(self.downloaded[s])   # the slot's previous irradiance has been read back
        rc.graph_launch(self.comp)
        self.solved[s].record(self.comp)
        self.down.wait_event(self.solved[s])
        rc.read_irradiance_async(out_ptr, self.down)
        self.downloaded[s].record(self.down)
        self.k += 1
        return s

    def done(self, slot: int) -> bool:
        return self.downloaded[slot].query()

    def wait(self):
        self.down.synchronize()

    def destroy(self):
        self.torch.cuda.synchronize()
        for rc in self.rcs:
            rc.destroy()
        self.rcs = []
