"""Serving loop for GI solves (no counterpart in the reference, which renders one frame per queue submit).

Requests are frames of resident scenes: (scene, time).  Each scene has moving rigid objects whose pose follows from
the time; a request poses them (vertex update), redraws the G-buffer, rebuilds the voxel clipmap and solves the
cascades on the device, and reads the irradiance back.

Continuous batching: requests that arrive while others are on the GPU are admitted as soon as a slot (a CUDA stream)
and their scene are free, and run concurrently with the requests already in flight; a scene is never solved by two
requests at once (its buffers are reused).  Residency: scenes stay on the device between requests; a request for a
scene that is not resident loads it if the HBM budget holds it, after evicting scenes that are idle, least recently
used first; otherwise it waits.  The plain loop serves the same requests one at a time in arrival order.

The scheduler talks to an executor (GpuExecutor on the device; tests also drive it with a simulated one), so the
admission and ordering logic runs without a GPU.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import configs, frame as fr, scenes
from .movers import MovingObjects, with_moving_boxes  # noqa: F401  (MovingObjects: re-exported)


@dataclass
class Request:
    rid: int
    scene: int
    t: float            # the frame's time (s): object poses follow from it
    arrival: float      # arrival time (s after the start of the stream)
    start: float = -1.0
    done: float = -1.0
    slot: int = -1

    @property
    def latency_ms(self) -> float:
        return 1000.0 * (self.done - self.arrival)


def poisson_arrivals(rate: float, n: int, n_scenes: int, seed: int = 1) -> List[Request]:
    """n requests of a Poisson stream of `rate` per second (numpy PCG64, seed 1), scenes uniform."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate, n)
    arr = np.cumsum(gaps) - gaps[0]
    sc = rng.integers(0, n_scenes, n)
    return [Request(i, int(sc[i]), float(arr[i]), float(arr[i])) for i in range(n)]


def serving_scene(spec: dict, n_objects: int):
    """A mixed scene of the batch distribution with n_objects moving boxes (sides 0.2-1 m, speeds 0-2 m/s)."""
    base = scenes.mixed_scene(spec["seed"], max(1000, spec["tris"] - 12 * n_objects))
    return with_moving_boxes(base, n_objects, scenes.PCG32(spec["seed"], stream=31))


@dataclass
class SceneSlot:
    spec: dict
    bytes: int = 0
    busy: bool = False
    last_used: float = 0.0


class Server:
    """Continuous-batching scheduler over an executor with `slots` concurrent streams and an HBM budget."""

    def __init__(self, executor, specs: List[dict], slots: int, hbm_budget: float):
        self.ex = executor
        self.specs = specs
        self.slots = slots
        self.budget = hbm_budget
        self.resident: Dict[int, SceneSlot] = {}
        self.stats = collections.Counter()

    def resident_bytes(self) -> int:
        return sum(s.bytes for s in self.resident.values())

    def _ensure_resident(self, sid: int, now: float) -> bool:
        if sid in self.resident:
            return True
        need = self.ex.scene_bytes(self.specs[sid])
        if need > self.budget:
            raise MemoryError(f"scene {sid} needs {need} bytes, more than the whole HBM budget {self.budget}")
        while self.resident_bytes() + need > self.budget:
            idle = [(s.last_used, k) for k, s in self.resident.items() if not s.busy]
            if not idle:
                return False
            _, victim = min(idle)
            self.ex.unload(victim)
            del self.resident[victim]
            self.stats["evictions"] += 1
        self.resident[sid] = SceneSlot(self.specs[sid], self.ex.load(sid, self.specs[sid]), False, now)
        self.stats["loads"] += 1
        return True

    def run(self, requests: List[Request], clock=None, on_done=None) -> dict:
        """Serves the requests (sorted by arrival) in real time; returns latency and throughput statistics.
        on_done(request, slot) runs at each completion, while the slot still holds the request's result."""
        clock = clock or _WallClock()
        pending: collections.deque = collections.deque()
        inflight: Dict[int, Request] = {}
        free = list(range(self.slots))
        nxt = 0
        done: List[Request] = []
        t0 = clock.start()
        while len(done) < len(requests):
            now = clock.now()
            while nxt < len(requests) and requests[nxt].arrival <= now:
                pending.append(requests[nxt])
                nxt += 1
            # completions free slots and scenes
            for slot, rq in list(inflight.items()):
                if self.ex.poll(slot):
                    rq.done = clock.now()
                    if on_done is not None:
                        on_done(rq, slot)
                    done.append(rq)
                    del inflight[slot]
                    free.append(slot)
                    self.resident[rq.scene].busy = False
                    self.resident[rq.scene].last_used = rq.done
            # admission: oldest first, skipping requests whose scene is busy or cannot be made resident yet
            if free and pending:
                keep = collections.deque()
                while pending and free:
                    rq = pending.popleft()
                    sc = self.resident.get(rq.scene)
                    if (sc is not None and sc.busy) or not self._ensure_resident(rq.scene, now):
                        keep.append(rq)
                        continue
                    slot = free.pop()
                    sc = self.resident[rq.scene]
                    sc.busy = True
                    rq.start, rq.slot = clock.now(), slot
                    self.ex.launch(slot, rq.scene, rq.t)
                    inflight[slot] = rq
                keep.extend(pending)
                pending = keep
            self.stats["max_pending"] = max(self.stats["max_pending"], len(pending))
            self.stats["max_inflight"] = max(self.stats["max_inflight"], len(inflight))
            if not inflight and not pending and nxt < len(requests):
                clock.sleep_until(requests[nxt].arrival)
            else:
                clock.idle()
        return summarize(done, dict(self.stats))


def plain_loop(executor, requests: List[Request], clock=None, on_done=None) -> dict:
    """The plain per-solve loop: one request at a time, in arrival order, on one stream."""
    clock = clock or _WallClock()
    clock.start()
    done = []
    for rq in requests:
        clock.sleep_until(rq.arrival)
        rq.start, rq.slot = clock.now(), 0
        executor.launch(0, rq.scene, rq.t)
        executor.wait(0)
        rq.done = clock.now()
        if on_done is not None:
            on_done(rq, 0)
        done.append(rq)
    return summarize(done, {})


def summarize(done: List[Request], extra: dict) -> dict:
    if not done:
        return {"completed": 0}
    lat = sorted(r.latency_ms for r in done)
    span = max(r.done for r in done) - min(r.arrival for r in done)
    p = lambda q: lat[min(len(lat) - 1, int(math.ceil(q * len(lat))) - 1)]
    return {"completed": len(done), "solves_per_s": len(done) / span if span > 0 else float("inf"),
            "p50_ms": p(0.5), "p99_ms": p(0.99), "max_ms": lat[-1], **extra}


class _WallClock:
    def start(self):
        self.t0 = time.perf_counter()
        return 0.0

    def now(self):
        return time.perf_counter() - self.t0

    def sleep_until(self, t):
        while self.now() < t:
            pass

    def idle(self):
        pass


class GpuExecutor:
    """Runs requests on the device: per slot a CUDA stream and a completion event; per resident scene its SceneGpu
    (moving objects as rigid bodies), VoxWorld, Rc (f16 atlases), pinned transform and result buffers, and one
    captured graph of the whole frame (pose, G-buffer, voxel rebuild, cascades, irradiance copy).  A request uploads
    its objects' transforms and launches the scene's graph: two calls."""

    def __init__(self, ctx, slots: int, atlas: str = "f16", n_objects=None, tuner=None):
        import torch
        from . import gpu
        self.torch, self.gpu = torch, gpu
        self.ctx = ctx
        self.atlas = atlas
        self.tuner = tuner          # an autotune.Autotuner: launch shapes picked per scene at load
        self.streams = [torch.cuda.Stream() for _ in range(max(1, slots))]
        self.events = [None] * len(self.streams)
        self.res: Dict[int, dict] = {}
        self.n_objects = n_objects or (lambda spec: 1 + int(scenes.PCG32(spec["seed"], stream=41).uniform(0, 200)))

    def scene_bytes(self, spec: dict) -> int:
        p, v = _params(spec, self.atlas)
        W, H = spec["width"], spec["height"]
        lay = configs.cascade_layout(p, W, H)
        elem = 16 if self.atlas == "f32" else 8
        rc = W * H * (4 + 8 + 16 + elem) + lay["probes_total"] * 52 + lay["rays_total"] * elem * 1
        vox = (v.levels * v.G ** 3 + v.maxBricks * (530 + 1) + 16 * (1 << 18) + 8 * (1 << 18) + v.maxVoxels * 6 + (1 << 20)) * 4
        return int(rc + vox + 140 * spec["tris"] + (4 << 20))

    def load(self, sid: int, spec: dict) -> int:
        torch = self.torch
        s, objs = serving_scene(spec, self.n_objects(spec))
        p, v = _params(spec, self.atlas)
        W, H = spec["width"], spec["height"]
        F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=s.sun_e, sky=s.sky,
                                         cascades=p.cascades, P=p.P))
        st = self.streams[0]
        sg = self.gpu.SceneGpu(self.ctx, s)
        sg.rigid_define(objs.first, objs.per, objs.centres.shape[0])
        vw = self.gpu.VoxWorld(sg, v)
        rc = self.gpu.Rc(self.ctx, p, W, H)
        rc.set_frame(F, st)
        vw.update(s.camera.eye)
        m = torch.empty((objs.centres.shape[0], 12), dtype=torch.float32).pin_memory()
        out = torch.empty(rc.irr_bytes(), dtype=torch.uint8).pin_memory()
        m.numpy()[:] = objs.transforms(0.0)
        sg.rigid_upload(m.data_ptr(), st)
        if self.tuner is not None:
            sg.rigid_apply(st)
            rc.render_gbuffer(sg, st)
            self.tuner.tune(rc, vw, st)
        rc.graph_capture_frame(vw, sg, out.data_ptr(), st)
        rc.graph_launch(st)
        st.synchronize()
        self.res[sid] = {"sg": sg, "vw": vw, "rc": rc, "objs": objs, "scene": s, "m": m, "out": out}
        return sg.bytes() + vw.bytes() + rc.bytes()

    def unload(self, sid: int):
        r = self.res.pop(sid)
        self.torch.cuda.synchronize()
        for k in ("rc", "vw", "sg"):
            r[k].destroy()

    def launch(self, slot: int, sid: int, t: float):
        r = self.res[sid]
        st = self.streams[slot]
        r["m"].numpy()[:] = r["objs"].transforms(t)
        r["sg"].rigid_upload(r["m"].data_ptr(), st)
        r["rc"].graph_launch(st)
        ev = self.torch.cuda.Event()
        ev.record(st)
        self.events[slot] = (ev, sid)

    def poll(self, slot: int) -> bool:
        e = self.events[slot]
        return e is None or e[0].query()

    def wait(self, slot: int):
        e = self.events[slot]
        if e is not None:
            e[0].synchronize()

    def result(self, slot: int) -> np.ndarray:
        """The irradiance (as stored) of the slot's last request; valid until its scene is launched again."""
        ev, sid = self.events[slot]
        ev.synchronize()
        return self.res[sid]["out"].numpy().copy()

    def destroy(self):
        for sid in list(self.res):
            self.unload(sid)


class PlainExecutor:
    """The plain per-solve path over a GpuExecutor's resident scenes: each request through the drop-in C-ABI calls
    one by one (transforms, pose, G-buffer, gi_solve, irradiance readback), no graph, on one stream."""

    def __init__(self, ex: GpuExecutor):
        self.ex = ex

    def launch(self, slot: int, sid: int, t: float):
        ex = self.ex
        r = ex.res[sid]
        st = ex.streams[0]
        r["m"].numpy()[:] = r["objs"].transforms(t)
        r["sg"].rigid_upload(r["m"].data_ptr(), st)
        r["sg"].rigid_apply(st)
        r["rc"].render_gbuffer(r["sg"], st)
        r["rc"].solve(r["vw"], st)
        r["rc"].read_irradiance_async(r["out"].data_ptr(), st)
        ev = ex.torch.cuda.Event()
        ev.record(st)
        ex.events[0] = (ev, sid)

    def poll(self, slot: int) -> bool:
        return self.ex.poll(0)

    def wait(self, slot: int):
        self.ex.wait(0)

    def result(self, slot: int) -> np.ndarray:
        return self.ex.result(0)


def _params(spec: dict, atlas: str):
    p = configs.parse_config(f"screen-8-voxel-{atlas}-dda256", {"cascades": spec["cascades"]})
    G, L = spec["G"], spec["levels"]
    v = configs.vox_params({"v0": spec["v0"], "levels": L, "G": G, "maxBricks": min(L * G ** 3, 32768),
                            "maxVoxels": 1 << 21})
    return p, v
