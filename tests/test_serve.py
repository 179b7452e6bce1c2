"""The serving loop: continuous batching under an HBM budget (scheduler checked on the CPU with a simulated executor
and clock), and on the GPU, every request's irradiance is the same served alone and served in a concurrent mix."""
import numpy as np
import pytest

from rtgi import scenes, serve


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def start(self):
        self.t = 0.0
        return 0.0

    def now(self):
        return self.t

    def sleep_until(self, t):
        self.t = max(self.t, t)

    def idle(self):
        self.t += 1e-4


class FakeExecutor:
    """Each solve takes 2 ms of simulated device time; scenes cost `scene_cost` bytes."""

    def __init__(self, clock, scene_cost=100):
        self.clock, self.cost = clock, scene_cost
        self.loaded, self.finish, self.log = set(), {}, []
        self.running = {}

    def scene_bytes(self, spec):
        return self.cost

    def load(self, sid, spec):
        assert sid not in self.loaded
        self.loaded.add(sid)
        self.log.append(("load", sid))
        return self.cost

    def unload(self, sid):
        assert sid not in self.running.values(), "evicted a scene with a solve in flight"
        self.loaded.remove(sid)
        self.log.append(("unload", sid))

    def launch(self, slot, sid, t):
        assert sid in self.loaded
        assert sid not in self.running.values(), "two solves of one scene at once"
        self.running[slot] = sid
        self.finish[slot] = self.clock.now() + 0.002

    def poll(self, slot):
        if self.clock.now() >= self.finish.get(slot, 0.0):
            self.running.pop(slot, None)
            return True
        return False

    def wait(self, slot):
        self.clock.t = max(self.clock.t, self.finish[slot])
        self.running.pop(slot, None)


def test_poisson_arrivals():
    rq = serve.poisson_arrivals(1000.0, 4000, 8)
    gaps = np.diff([r.arrival for r in rq])
    assert abs(gaps.mean() - 1e-3) < 1e-4 and rq[0].arrival == 0.0
    assert {r.scene for r in rq} == set(range(8))


def test_scheduler_overlaps_and_respects_budget():
    clock = FakeClock()
    ex = FakeExecutor(clock, scene_cost=100)
    specs = [scenes.batch_spec(s) for s in range(6)]
    srv = serve.Server(ex, specs, slots=4, hbm_budget=350)      # at most 3 scenes resident
    reqs = serve.poisson_arrivals(2000.0, 300, 6)
    st = srv.run(reqs, clock)
    assert st["completed"] == 300
    assert st["max_inflight"] > 1                                 # requests overlapped on the device
    assert st["evictions"] > 0 and len(ex.loaded) <= 3
    loads = [k for k, _ in ex.log if k == "load"]
    assert st["loads"] == len(loads)
    # served faster than the plain one-at-a-time loop on the same stream of requests
    clock2 = FakeClock()
    ex2 = FakeExecutor(clock2)
    for s in range(6):
        ex2.load(s, specs[s])
    plain = serve.plain_loop(ex2, serve.poisson_arrivals(2000.0, 300, 6), clock2)
    assert plain["p99_ms"] > st["p99_ms"]


def test_scheduler_rejects_scene_larger_than_budget():
    clock = FakeClock()
    srv = serve.Server(FakeExecutor(clock, scene_cost=1000), [scenes.batch_spec(0)], slots=2, hbm_budget=500)
    with pytest.raises(MemoryError):
        srv.run(serve.poisson_arrivals(100.0, 3, 1), clock)


def test_moving_objects_pose():
    spec = dict(scenes.batch_spec(5), tris=6000)
    s, objs = serve.serving_scene(spec, 7)
    p0, n0 = objs.pose(0.0)
    assert np.allclose(p0, s.positions[objs.first:], atol=1e-5)
    p1, n1 = objs.pose(1.0)
    assert p1.shape == p0.shape and not np.allclose(p1, p0)
    assert np.allclose(np.linalg.norm(n1, axis=1), 1.0, atol=1e-5)


@pytest.mark.gpu
def test_served_result_same_alone_and_in_mix():
    import torch
    from rtgi import gpu
    ctx = gpu.Context(0)
    specs = []
    for s in range(4):
        sp = scenes.batch_spec(200 + s)
        sp["tris"] = min(sp["tris"], 40_000)
        sp["width"], sp["height"] = min(sp["width"], 640), min(sp["height"], 360)
        specs.append(sp)
    ex = serve.GpuExecutor(ctx, slots=4, n_objects=lambda spec: 25)
    for i, sp in enumerate(specs):
        ex.load(i, sp)
    probe = serve.Request(0, 2, 0.37, 0.0)
    alone = {}
    serve.plain_loop(ex, [probe], on_done=lambda rq, slot: alone.setdefault(rq.rid, ex.result(slot)))
    reqs = serve.poisson_arrivals(3000.0, 60, 4)
    reqs[30].scene, reqs[30].t = 2, 0.37          # the same frame, now in a mix of concurrent requests
    mixed = {}
    srv = serve.Server(ex, specs, slots=4, hbm_budget=150e9)
    srv.resident = {i: serve.SceneSlot(sp, 1) for i, sp in enumerate(specs)}
    st = srv.run(reqs, on_done=lambda rq, slot: mixed.setdefault(rq.rid, ex.result(slot)) if rq.rid == 30 else None)
    assert st["completed"] == 60 and st["max_inflight"] >= 2
    assert np.array_equal(mixed[30], alone[0]), "a request's result changed when served in the mix"
    # the plain path (the C-ABI calls one by one, no graph) computes the same frame identically
    plain = {}
    serve.plain_loop(serve.PlainExecutor(ex), [serve.Request(1, 2, 0.37, 0.0)],
                     on_done=lambda rq, slot: plain.setdefault(rq.rid, ex.result(slot)))
    assert np.array_equal(plain[1], alone[0])
    assert np.any(alone[0] != 0)
    ex.destroy()
    ctx.destroy()
