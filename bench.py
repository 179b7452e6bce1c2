#!/usr/bin/env python
"""GI solves/s of the B200 path on the large procedural workload (the colonnade: ~260k triangles, a clipmap of
4 levels of 128^3 voxels from 0.1 m, 5 radiance cascades at 1920x1080, DDA capped at 256 steps, f32 atlases).

A step is one GI solve: the voxel clipmap rebuild from the triangles (voxel.ts VOX_STAGES) and the cascades
(giBuild setupScreen, giTrace, giMerge + projectSH, giGather), replayed from one captured CUDA graph.  Inputs (scene,
frame, G-buffer) are resident in HBM; L2 is flushed (a 256 MiB write) between steps, outside the step's events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload colonnade|room]

One process per GPU (torchrun for N > 1); every rank solves its own replica (no data-path collective), the job's
value is all ranks' solves over the slowest rank's device time.  Rank 0 prints one JSON line.
``--impl reference`` times the reference's algorithm on the host cores instead: the reference itself (TypeScript +
WGSL through Dawn) cannot run here, so its CPU restatement (oracle/) runs with every host thread.
"""
import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "real-time-gi-lab_b200"))

import numpy as np

METRIC = "GI solves/s & p99 ms (served batch vs plain), DDA steps/s, % HBM roofline"


def workload(name):
    from rtgi import configs, frame as fr, scenes
    if name == "colonnade":
        s = scenes.colonnade_scene(0)
        W, H = 1920, 1080
        p = configs.parse_config("screen-8-voxel-f32-dda256-irr16", {"cascades": 5})
        v = configs.vox_params({"v0": 0.1, "levels": 4, "G": 16, "maxBricks": 16384, "maxVoxels": 1 << 22})
        sun_e, sky = s.sun_e, s.sky
        shadow = fr.SHADOW_SIZE   # the sun's shadow map over the scene (voxSun in every rebuild)
    else:
        s = scenes.room_scene(0)
        W, H = 256, 256
        p = configs.parse_config("screen-8-voxel-f32-dda64-irr16", {"cascades": 2})
        v = configs.vox_params({"v0": 0.16, "levels": 1, "G": 8, "maxBricks": 512, "maxVoxels": 1 << 18})
        sun_e, sky = (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)
        shadow = 0                # sun off
    lvp, bias = [0.0] * 16, (0.0, 0.0)
    if shadow:
        bmin, bmax = fr.scene_bounds(s.positions)
        lvp, bias = fr.scene_sun_view_proj(bmin, bmax, s.sun_dir), fr.SHADOW_BIAS
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=sun_e, sky=sky,
                                     cascades=p.cascades, P=p.P, light_view_proj=lvp, shadow_bias=bias))
    desc = {"workload": f"{name}: {s.triangle_count} triangles, clipmap {v.levels} x {v.G * 8}^3 voxels from "
                        f"{v.v0} m, {p.cascades} cascades at {W}x{H}, DDA cap {p.ddaCap}, atlas {p.atlas}, "
                        f"irradiance {'rgba16float' if p.irr16 else 'rgba32float'}",
            "triangles": s.triangle_count, "resolution": [W, H], "cascades": p.cascades, "levels": v.levels,
            "G": v.G, "v0": v.v0, "dda_cap": p.ddaCap, "atlas": p.atlas, "method": "screen-8-voxel",
            "irradiance": "rgba16float, the reference's rc.irr format (rc.ts:1073); every pass before the store in f32"
                          if p.irr16 else "rgba32float",
            "shadow_map": shadow}
    if shadow:
        desc["workload"] += f", sun shadow map {shadow}^2"
    return s, W, H, p, v, F, desc


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.proc, self.path = device, None, None

    def start(self):
        try:
            import tempfile
            self.path = tempfile.mktemp(suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, t0=None, t1=None):
        """Summary of the samples taken between wall-clock times t0 and t1 (all samples when none fall there)."""
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [l.split(", ") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        if t0 is not None:
            import datetime
            def ts(r):
                try:
                    return datetime.datetime.strptime(r[0].strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except Exception:
                    return None
            inside = [r for r in rows if ts(r) is not None and t0 <= ts(r) <= t1]
            if inside:
                rows = inside
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def measured_peak():
    try:
        m = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(name):
    """DRAM bytes per launch of the trace kernel from the committed ncu summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", f"ncu_trace_{name}.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def trace_algorithmic_bytes(rc_layout, hdr, vox):
    """Compulsory bytes of one giTrace launch: probes read (48 B each), the atlas written (16 B per ray in f32), the
    clipmap read once (brick pointers, occupancy + first attribute per brick, 16-byte attribute record + sun
    visibility per voxel)."""
    nb = int(min(hdr[0], vox.maxBricks))
    nv = int(min(hdr[1], vox.maxVoxels))
    elem = 16 if rc_layout["atlas"] == 0 else 8
    return (48 * rc_layout["probes_total"] + elem * rc_layout["rays_total"] + 4 * vox.levels * vox.G ** 3
            + 68 * nb + 20 * nv)


def cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow=None):
    st = bind.vox_build(s, v.v0, v.levels, v.G, v.maxBricks, v.maxVoxels, s.camera.eye)
    if shadow is not None:
        bind.vox_sun(st, F, shadow)
    bind.rc_solve(st, lay, F, depth, normal)


def cpu_baseline(s, v, p, F, depth, normal, shadow_size=0, budget_s=8.0, min_solves=2):
    """The oracle (a CPU restatement of the reference's shaders) timed on this host's cores, bounded samples: every
    pass on all host threads (the voxel passes' triangle loops, the rays and the pixels), then the same on one."""
    from oracle import bind
    from rtgi import configs
    lay = configs.cascade_layout(p, depth.shape[1], depth.shape[0])
    shadow = bind.shadow_render(s, F, shadow_size) if shadow_size else None   # an input, as the G-buffer

    def leg(threads):
        old = os.environ.get("ORC_THREADS")
        if threads:
            os.environ["ORC_THREADS"] = str(threads)
        try:
            cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow)   # warm
            n, t0 = 0, time.perf_counter()
            while n < min_solves or time.perf_counter() - t0 < budget_s:
                cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow)
                n += 1
            return n, time.perf_counter() - t0
        finally:
            if old is None:
                os.environ.pop("ORC_THREADS", None)
            else:
                os.environ["ORC_THREADS"] = old

    cores = int(os.environ.get("ORC_THREADS", os.cpu_count() or 1))
    n, dt = leg(None)
    n1, dt1 = leg(1)
    return {"value": n / dt, "unit": "solves/s", "cores": cores, "kind": "port", "cores_1_value": n1 / dt1,
            "sample": f"{n} full solves of the workload (voxel rebuild + setup/trace/merge/SH/gather; the rebuild's "
                      f"triangle passes, the rays and the pixels on {cores} threads) in {dt:.1f} s; 1 thread: {n1} "
                      f"solves in {dt1:.1f} s"}


def run_batched(args, ctx, stream, flush):
    """The uneven batch (64 seeded specs): every solve replayed alone from its own graph, one after another, with the
    default launch shapes and with the autotuner's, and all of them (autotuned) as one batch graph of parallel solve
    chains.  Device time with CUDA events, L2 flushed between replays."""
    import collections
    import torch
    from rtgi import autotune, batch, scenes
    specs = [scenes.batch_spec(s) for s in range(args.batch)]
    solves = [batch.make_solve(ctx, sp, stream=stream) for sp in specs]
    reps = 5
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def time_alone():
        for x in solves:
            x.rc.graph_capture(x.vox, stream)
        with torch.cuda.stream(stream):
            for x in solves:   # warm-up
                x.rc.graph_launch(stream)
            per = [[] for _ in solves]
            for _ in range(reps):
                for i, x in enumerate(solves):
                    flush.zero_()
                    e0, e1 = ev(), ev()
                    e0.record(stream)
                    x.rc.graph_launch(stream)
                    e1.record(stream)
                    per[i].append((e0, e1))
            torch.cuda.synchronize()
        return [statistics.median(a.elapsed_time(c) for a, c in per[i]) for i in range(len(solves))]

    alone_default = time_alone()
    t0 = time.perf_counter()
    tuner = autotune.Autotuner(reps=3)
    picks = [tuner.tune(x.rc, x.vox, stream) for x in solves]
    tune_s = time.perf_counter() - t0
    alone_ms = time_alone()
    b = batch.make_batch(ctx, solves, stream)
    with torch.cuda.stream(stream):
        b.launch(stream)
        stream.synchronize()
        bt = []
        for _ in range(reps * 4):
            flush.zero_()
            e0, e1 = ev(), ev()
            e0.record(stream)
            b.launch(stream)
            e1.record(stream)
            bt.append((e0, e1))
        torch.cuda.synchronize()
    batch_ms = sorted(a.elapsed_time(c) for a, c in bt)
    # the same solves pass by pass: rebuilds in parallel, then one launch per cascade pass over all of them
    b.capture_passes(stream)
    with torch.cuda.stream(stream):
        b.launch(stream)
        stream.synchronize()
        bp = []
        for _ in range(reps * 4):
            flush.zero_()
            e0, e1 = ev(), ev()
            e0.record(stream)
            b.launch(stream)
            e1.record(stream)
            bp.append((e0, e1))
        torch.cuda.synchronize()
    passes_ms = sorted(a.elapsed_time(c) for a, c in bp)
    chosen = collections.Counter()
    for pk in picks:
        for k, val in list(pk["rc"].items()) + list(pk["vox"].items()):
            chosen[f"{k}={val}"] += 1
    out = {"solves": len(solves), "triangles": sum(x.scene.triangle_count for x in solves),
           "rays": sum(x.rc.layout["rays_total"] for x in solves),
           "plain_solves_per_s": len(solves) / (sum(alone_default) / 1000.0),
           "plain_tuned_solves_per_s": len(solves) / (sum(alone_ms) / 1000.0),
           "plain_p50_ms": statistics.median(alone_default), "plain_p99_ms": sorted(alone_default)[-1],
           "batch_ms_p50": statistics.median(batch_ms), "batch_ms_p99": batch_ms[-1],
           "batched_solves_per_s": len(solves) / (statistics.median(batch_ms) / 1000.0),
           "passes_ms_p50": statistics.median(passes_ms), "passes_ms_p99": passes_ms[-1],
           "batched_passes_solves_per_s": len(solves) / (statistics.median(passes_ms) / 1000.0),
           "autotune_s": tune_s, "autotune_choices": dict(sorted(chosen.items())),
           "mode": "one CUDA graph of parallel per-solve kernel chains (gi_batch_capture), launch shapes from the "
                   "autotuner; passes: the rebuilds as parallel branches, then one launch per cascade pass over all "
                   "64 solves (gi_batch_capture_passes)",
           "spec": "scenes.batch_spec(0..63): tris log-U(5k, 500k), G 4..32 x 1-4 levels, 320x180..1920x1080, 2-5 cascades"}
    out["speedup"] = out["batched_solves_per_s"] / out["plain_solves_per_s"]
    out["speedup_vs_tuned_plain"] = out["batched_solves_per_s"] / out["plain_tuned_solves_per_s"]
    b.destroy()
    for x in solves:
        x.destroy()
    return out


def run_precision(args, ctx):
    """Irradiance error of the f32/f16/bf16 atlases against the FP64 merge + gather, colonnade with 64 moving boxes,
    clipmap rebuilt every frame (rtgi.precision)."""
    from rtgi import precision
    t0 = time.time()
    r = precision.run(ctx, frames=args.precision_frames)
    r["wall_s"] = time.time() - t0
    return r


def run_served(args, ctx, rank=0, world=1):
    """The serving loop (continuous batching, 8 slots, HBM budget 150 GB, f16 atlases) against the plain one-at-a-time
    loop, on Poisson request streams at several rates over 12 resident scenes of the batch distribution, each with
    1-200 moving objects.  Latency = arrival to irradiance in host memory (host wall clock).  On N GPUs the stream's
    rate is the whole job's: requests are routed to the ranks owning their scenes (rtgi.route), each rank serves its
    share, and the statistics pool every rank's requests."""
    from rtgi import autotune, route, scenes, serve
    specs = [scenes.batch_spec(1000 + s) for s in range(12)]
    ex = serve.GpuExecutor(ctx, slots=8, atlas="f16", tuner=autotune.Autotuner(reps=3))
    srv = serve.Server(ex, specs, slots=8, hbm_budget=150e9)
    rs = route.RoutedServer(lambda mine: srv, specs, rank, world)
    for i in rs.mine:   # this rank's scenes resident before the streams start
        srv._ensure_resident(i, 0.0)
    plain = serve.PlainExecutor(ex)
    served = lambda reqs: rs.run(reqs)
    plained = lambda reqs: rs.run_with(lambda mine, clock: serve.plain_loop(plain, mine, clock), reqs)
    # warm-up of both paths (every slot's stream)
    plained(serve.poisson_arrivals(1000.0 * world, 24 * world, len(specs), seed=7))
    served(serve.poisson_arrivals(4000.0 * world, 64 * world, len(specs), seed=7))
    rates = []
    for rate in args.serve_rates:
        n = int(min(args.serve_max, max(50, rate * args.serve_seconds)))
        st = served(serve.poisson_arrivals(rate, n, len(specs)))
        pl = plained(serve.poisson_arrivals(rate, n, len(specs)))
        rates.append({"rate": rate, "requests": n, "served": st, "plain": pl,
                      "throughput_ratio": st["solves_per_s"] / pl["solves_per_s"]})
    # the criterion as worded: per path the highest sustained rate whose p99 stays within a budget, on a rate grid
    # (every lower rate of the grid within the budget too), and the ratio of the two paths at each budget
    grid = [200, 300, 450, 650, 900, 1250, 1700, 2300, 3100, 4200, 5600]
    sweep = {"served": [], "plain": []}
    for rate in grid:
        n = int(min(args.serve_max, max(200, rate * 0.5)))
        sweep["served"].append((rate, served(serve.poisson_arrivals(rate, n, len(specs), seed=11))))
        sweep["plain"].append((rate, plained(serve.poisson_arrivals(rate, n, len(specs), seed=11))))
    budgets = {}
    for b in (2.0, 5.0):
        best = {}
        for path, runs in sweep.items():
            ok = None
            for rate, r in runs:
                if r["p99_ms"] > b:
                    break
                ok = {"rate": rate, "solves_per_s": r["solves_per_s"], "p99_ms": r["p99_ms"]}
            best[path] = ok
        ratio = (best["served"]["solves_per_s"] / best["plain"]["solves_per_s"]
                 if best["served"] and best["plain"] else None)
        budgets[f"p99<={b:g}ms"] = {**best, "ratio": ratio}
    res_bytes = srv.resident_bytes()
    ex.destroy()
    return {"scenes": len(specs), "slots": 8, "atlas": "f16", "hbm_budget_bytes": 150e9, "resident_bytes": res_bytes,
            "ranks": world, "owners": rs.owners,
            "objects_per_scene": [ex.n_objects(sp) for sp in specs], "rates": rates,
            "ratio_at_p99_budget": budgets,
            "sweep": {path: [{"rate": rate, "solves_per_s": r["solves_per_s"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"]}
                             for rate, r in runs] for path, runs in sweep.items()},
            "latency": "arrival -> irradiance in pinned host memory, host wall clock",
            "request": "upload object transforms, pose objects on the device, G-buffer, voxel rebuild, cascades, "
                       "irradiance readback (f16)",
            "served_path": "8 streams, continuous batching, one captured graph per scene (whole frame)",
            "plain_path": "one request at a time on one stream through the C-ABI calls (no graph)"}


def run_reference(args, rank):
    """The reference's algorithm on the host cores (oracle/), on the same workload, config and metric."""
    if rank != 0:
        return
    from oracle import bind
    from rtgi import configs
    s, W, H, p, v, F, desc = workload(args.workload)
    depth, normal, _ = bind.raster_gbuffer(s, F, W, H)   # inputs, not timed
    shadow = bind.shadow_render(s, F, desc["shadow_map"]) if desc["shadow_map"] else None
    lay = configs.cascade_layout(p, W, H)
    for _ in range(args.warmup):
        cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow)
    # a bounded sample: at most ~90 s of solves
    t_one = time.perf_counter()
    cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow)
    t_one = time.perf_counter() - t_one
    k = max(1, min(args.steps, int(90.0 / max(t_one, 1e-3))))
    times = []
    for _ in range(k):
        t0 = time.perf_counter()
        cpu_solve_once(bind, s, v, lay, F, depth, normal, shadow)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = k / total
    cores = int(os.environ.get("ORC_THREADS", os.cpu_count() or 1))
    times.sort()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": k, "warmup": args.warmup, "ms_per_step": 1000 * total / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {**desc, "parallelism": "host threads"},
            "p50_ms": 1000 * times[len(times) // 2], "p99_ms": 1000 * times[min(len(times) - 1, int(0.99 * len(times)))],
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{k} of the requested {args.steps} steps (each one full solve; bounded to ~90 s); "
                                       "the reference itself (WGSL through Dawn on Node) cannot run on this host"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def init_ranks(world: int, backend: str = "nccl", timeout_s: float = 120.0):
    """torch.distributed for N > 1 replicas (env rendezvous: MASTER_ADDR/PORT, RANK, WORLD_SIZE), else None."""
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x: float, dist, device) -> float:
    """The largest x of all ranks (every rank takes part; device: where the backend's tensors live)."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rebuild_launches(levels: int) -> int:
    """Kernels of one voxel rebuild (gi_launch_vox_build): clear, markBricks and its big items, allocBricks, the brick
    init, voxBits and its big items, reduce (more than one level), allocVoxels, resolveAttr."""
    return 9 + (1 if levels > 1 else 0)


def whole_job_rate(units_per_rank: float, max_seconds: float, world: int) -> float:
    """Units all ranks processed over the slowest rank's time (replicas: weak scaling)."""
    return world * units_per_rank / max_seconds


def run_world_items(args, ctx, stream):
    """Worlds (world.ts): the room scene placed at 121 instances 12 m apart (a 130 m town of 292k triangles) read by the
    voxel rebuild as per-frame work items (chunks inside the windows, clustered copies at the coarse levels), against
    the same geometry baked into one flat scene that the rebuild reads whole.  Device time of the rebuild alone."""
    import dataclasses
    import torch
    from rtgi import configs, gpu, scenes, world as W
    room = scenes.room_scene(0)
    v = configs.vox_params({"v0": 0.08, "levels": 4, "G": 16, "maxBricks": 32768, "maxVoxels": 1 << 22})
    inst = [(12.0 * i, 0.0, 12.0 * j) for j in range(-5, 6) for i in range(-5, 6)]
    inst.remove((0.0, 0.0, 0.0))
    inst.insert(0, (0.0, 0.0, 0.0))
    s2, w = W.with_world(room, inst, float(v.v0), v.levels)
    P = np.asarray(room.positions, np.float32)
    flat_pos = np.concatenate([P + np.asarray(o, np.float32) for o in inst])
    flat_tri = np.concatenate([room.tri.astype(np.int64) + np.array([k * P.shape[0]] * 3 + [0]) for k in range(len(inst))])
    flat = dataclasses.replace(room, positions=flat_pos, normals=np.concatenate([room.normals] * len(inst)),
                               tri=flat_tri.astype(np.uint32))
    eye = room.camera.eye
    out = {"instances": len(inst), "triangles_per_instance": room.triangle_count,
           "clipmap": f"{v.levels} x {v.G * 8}^3 voxels from {v.v0} m"}
    for name, scene, world in (("items", s2, w), ("flat", flat, None)):
        sg = gpu.SceneGpu(ctx, scene)
        vw = gpu.VoxWorld(sg, v)
        if world is not None:
            vw.set_world(world)
        vw.update(eye)
        with torch.cuda.stream(stream):
            for _ in range(5):
                vw.encode(stream)
            ms = []
            for _ in range(50):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                vw.encode(stream)
                e1.record(stream)
                ms.append((e0, e1))
            torch.cuda.synchronize()
        hdr = vw.read_counters(stream)["hdr"]
        out[name] = {"rebuild_ms": statistics.median(a.elapsed_time(b) for a, b in ms),
                     "bricks": int(hdr[0]), "voxels": int(hdr[1])}
        if world is not None:
            items = W.select_items(world, W.windows(float(v.v0), v.levels, v.G, eye))
            out[name].update(items=len(items), threads=sum(it.count for it in items),
                             items_per_level=[sum(1 for it in items if it.start == L) for L in range(v.levels)])
        else:
            out[name]["threads"] = scene.triangle_count
        vw.destroy()
        sg.destroy()
    return out


def run_dynamic(args, ctx, stream, flush, dist, world):
    """The dynamic layer (dynlayer.ts) on the colonnade with 64 moving boxes as the scene's dynamic tail: the static rows
    rebuilt into the clipmap, the boxes splatted into the layer, the cascades reading it (traceDyn), solves replayed from
    one graph; against the same solve with the layer unbound (the boxes then absent).  With multi-bounce on, the layer
    (with its albedo words) without and with the token obj (the boxes receive the bounce volume's light and block and
    reflect its rays: dynInject, bnTraceDyn).  Device time, L2 flushed between steps outside the step events."""
    import torch
    from rtgi import frame as fr, gpu, movers, scenes
    s0, W, H, p, v, F0, desc = workload(args.workload)
    s, objs = movers.with_moving_boxes(s0, 64, scenes.PCG32(2, stream=9), area=(0.0, 0.0, 12.0, 12.0))
    first = s0.triangle_count
    bmin, bmax = fr.scene_bounds(s.positions)
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=s.sun_e, sky=s.sky,
                                     cascades=p.cascades, P=p.P, light_view_proj=fr.scene_sun_view_proj(bmin, bmax, s.sun_dir),
                                     shadow_bias=fr.SHADOW_BIAS))
    sg = gpu.SceneGpu(ctx, s)
    sg.set_static_count(first)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    dyn = gpu.DynLayer(vw, first, bricks=2048)
    dyn_alb = gpu.DynLayer(vw, first, bricks=2048, albedo=True)
    out = {"objects": 64, "dynamic_triangles": s.triangle_count - first, "bricks_pool": 2048}
    with torch.cuda.stream(stream):
        rc.set_frame(F, stream)
        rc.render_gbuffer(sg, stream)
        rc.render_shadow(sg, desc["shadow_map"] or 4096, stream)
        vw.update(s.camera.eye)
        for name, layer, bounce, objects in (("with_layer", dyn, False, False), ("without", None, False, False),
                                             ("bounce_with_layer", dyn_alb, True, False),
                                             ("bounce_objects", dyn_alb, True, True)):
            rc.set_dyn(layer)
            rc.set_bounce(vw if bounce else None)
            rc.set_objects(objects)
            rc.set_timing(True)
            pm = {k: [] for k in rc.PASSES}
            for _ in range(max(5, args.warmup)):
                rc.solve(vw, stream)
                for k, x in rc.pass_times().items():
                    pm[k].append(x)
            rc.set_timing(False)
            rc.graph_capture(vw, stream)
            n = max(3, min(args.steps, 200))
            es, ee = ([torch.cuda.Event(enable_timing=True) for _ in range(n)] for _ in range(2))
            for k in range(n):
                flush.zero_()
                es[k].record(stream)
                rc.graph_launch(stream)
                ee[k].record(stream)
            torch.cuda.synchronize()
            ms = sorted(a.elapsed_time(b) for a, b in zip(es, ee))
            tot = max_over_ranks(sum(ms), dist, "cuda")
            out[name] = {"value": whole_job_rate(n, tot / 1000.0, world), "unit": "solves/s", "ms_per_step": tot / n,
                         "passes_ms": {k: statistics.median(x) for k, x in pm.items()}}
        out["layer"] = {k: val for k, val in dyn.read_counters(stream).items() if k != "hdr"}
    rc.set_dyn(None)
    rc.set_bounce(None)
    for h in (rc, dyn, dyn_alb, vw, sg):
        h.destroy()
    return out


def run_world(args, ctx, stream, sg, vw, s, W, H, v, desc, flush, dist, world):
    """World probes (gi_rc_create_world) on the workload's scene and clipmap: the config world-48-voxel-rc2-vrel-f32
    with the default capacities, solves replayed from one graph (the c0 history carries between them), L2 flushed
    between steps outside the step events."""
    import torch
    from rtgi import _lib, configs, frame as fr, gpu
    p = configs.parse_config("world-48-voxel-rc2-vrel-f32-dda256", {"cascades": 5})
    lvp, bias = [0.0] * 16, (0.0, 0.0)
    if desc["shadow_map"]:
        bmin, bmax = fr.scene_bounds(s.positions)
        lvp, bias = fr.scene_sun_view_proj(bmin, bmax, s.sun_dir), fr.SHADOW_BIAS
    F = fr.pack_frame(fr.FrameParams(cam=s.camera, width=W, height=H, sun_dir=s.sun_dir, sun_e=s.sun_e, sky=s.sky,
                                     cascades=p.cascades, P=p.P, light_view_proj=lvp, shadow_bias=bias))
    rc = gpu.Rc(ctx, p, W, H)
    with torch.cuda.stream(stream):
        rc.set_frame(F, stream)
        rc.render_gbuffer(sg, stream)
        if desc["shadow_map"]:
            rc.render_shadow(sg, desc["shadow_map"], stream)
        vw.update(s.camera.eye)
        rc.set_stats(1)
        rc.solve(vw, stream)
        counts = rc.read_counts(stream)
        rc.set_stats(0)
        rc.set_timing(True)
        w_pass = {k: [] for k in rc.PASSES}
        for _ in range(max(5, args.warmup)):
            rc.solve(vw, stream)
            for k, x in rc.pass_times().items():
                w_pass[k].append(x)
        rc.set_timing(False)
        rc.graph_capture(vw, stream)
        for _ in range(args.warmup):
            flush.zero_()
            rc.graph_launch(stream)
        n_w = max(3, min(args.steps, 500))
        ws_, we_ = ([torch.cuda.Event(enable_timing=True) for _ in range(n_w)] for _ in range(2))
        for k in range(n_w):
            flush.zero_()
            ws_[k].record(stream)
            rc.graph_launch(stream)
            we_[k].record(stream)
        torch.cuda.synchronize()
        counts2 = rc.read_counts(stream)
    w_ms = sorted(a.elapsed_time(c) for a, c in zip(ws_, we_))
    w_total = max_over_ranks(sum(w_ms), dist, "cuda")
    # the reference renderer's default transport: the same with multi-bounce on (rc.ts:90)
    with torch.cuda.stream(stream):
        rc.set_bounce(vw)
        rc.set_timing(True)
        b_pass = {k: [] for k in rc.PASSES}
        for _ in range(max(5, args.warmup)):
            rc.solve(vw, stream)
            for k, x in rc.pass_times().items():
                b_pass[k].append(x)
        rc.set_timing(False)
        rc.graph_capture(vw, stream)
        bs, be = ([torch.cuda.Event(enable_timing=True) for _ in range(n_w)] for _ in range(2))
        for k in range(n_w):
            flush.zero_()
            bs[k].record(stream)
            rc.graph_launch(stream)
            be[k].record(stream)
        torch.cuda.synchronize()
        rc.set_bounce(None)
    b_ms = sorted(a.elapsed_time(c) for a, c in zip(bs, be))
    b_total = max_over_ranks(sum(b_ms), dist, "cuda")
    lay = rc.layout
    probes = [int(min(counts[c], lay["casc"][c]["cap"])) for c in range(p.cascades)]
    rays = sum(n * lay["casc"][c]["res"] ** 2 for c, n in enumerate(probes))
    valid = int((rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32) > 0).sum())
    out = {"value": whole_job_rate(n_w, w_total / 1000.0, world), "unit": "solves/s", "steps": n_w,
           "ms_per_step": w_total / n_w, "p50_ms": w_ms[n_w // 2],
           "p99_ms": w_ms[min(n_w - 1, int(math.ceil(0.99 * n_w)) - 1)],
           "config": "world-48-voxel-rc2-vrel-f32-dda256, 5 cascades, caps 2^18 .. 2^11, the same clipmap and shadow map",
           "passes_ms": {k: statistics.median(x) for k, x in w_pass.items()},
           "probes": probes, "rays": rays, "dda_steps": int(counts[32:32 + p.cascades].sum()),
           "black_pixels_pct": 100.0 * float(counts2[72:80].sum()) / max(valid, 1),
           "bounce": {"value": whole_job_rate(n_w, b_total / 1000.0, world), "unit": "solves/s",
                      "ms_per_step": b_total / n_w, "p99_ms": b_ms[min(n_w - 1, int(math.ceil(0.99 * n_w)) - 1)],
                      "passes_ms": {k: statistics.median(x) for k, x in b_pass.items()}},
           # voxel rebuild, then clear, registerPixels, the paired compact / relocateVox / registerUp / linkParents
           # launches (2N + 1 with voxel relocation), the trace, a merge per cascade, projectSH, the gather
           "gpu_launches_per_solve": rebuild_launches(v.levels) + 2 + 2 * p.cascades + 1 + 1 + p.cascades + 2}
    rc.destroy()
    return out


def run_e2e(ctx, vw, p, W, H, F, host, shadow, tuned, n, dist, world, slots=2):
    """host: (frame, depth, normal) pinned tensors; a normal tensor of 3 halves per pixel is uploaded as rgb16f."""
    """Solves/s through rtgi.pipeline with host buffers: every step uploads its frame and G-buffer from pinned memory
    and downloads its irradiance into pinned memory, the copies of neighbouring frames overlapping the solve."""
    import torch
    from rtgi import pipeline
    frame_h, depth_h, normal_h = host
    rgb = normal_h.numel() == 3 * W * H
    pipe = pipeline.FramePipeline(ctx, vw, p, W, H, F, depth_h.data_ptr(), normal_h.data_ptr(), slots=slots,
                                  shadow=shadow, tuning=tuned["rc"], normal_rgb=rgb)
    irr_h = [torch.empty(pipe.irr_bytes, dtype=torch.uint8).pin_memory() for _ in range(slots)]
    for k in range(2 * slots):
        pipe.submit(frame_h.data_ptr(), depth_h.data_ptr(), normal_h.data_ptr(), irr_h[k % slots].data_ptr())
    pipe.wait()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for k in range(n):
        pipe.submit(frame_h.data_ptr(), depth_h.data_ptr(), normal_h.data_ptr(), irr_h[k % slots].data_ptr())
    pipe.wait()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - e0
    pipe.destroy()
    value = whole_job_rate(n, max_over_ranks(e2e_s, dist, "cuda"), world)
    if dist:
        dist.barrier()
    return {"value": value, "unit": "solves/s",
            "h2d_bytes_per_step": int(depth_h.numel() * 4 + normal_h.numel() * 2 + frame_h.numel() * 4),
            "d2h_bytes_per_step": int(irr_h[0].numel()), "steps": n,
            "irradiance": "rgba16float" if p.irr16 else "rgba32float",
            "normal_upload": "rgb16f (3 halves per pixel)" if rgb else "rgba16f",
            "mode": f"rtgi.pipeline: copies of neighbouring frames overlap the solve ({slots} cascade sets); wall "
                    "clock around the steps, max over ranks"}


def run_ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = init_ranks(world)
    from rtgi import _lib, configs, gpu

    s, W, H, p, v, F, desc = workload(args.workload)
    stream = torch.cuda.Stream()
    ctx = gpu.Context(local_rank)
    sg = gpu.SceneGpu(ctx, s)
    vw = gpu.VoxWorld(sg, v)
    rc = gpu.Rc(ctx, p, W, H)
    with torch.cuda.stream(stream):
        rc.set_frame(F, stream)
        rc.render_gbuffer(sg, stream)
        shadow_ms = None
        if desc["shadow_map"]:   # an input of the solve, as the G-buffer: drawn once (static scene and sun)
            rc.render_shadow(sg, desc["shadow_map"], stream)   # warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc.render_shadow(sg, desc["shadow_map"], stream)
            e1.record(stream)
            stream.synchronize()
            shadow_ms = e0.elapsed_time(e1)
        vw.update(s.camera.eye)
        # DDA work of one solve (steps counted as rc.ts:232-235)
        rc.set_stats(1)
        rc.solve(vw, stream)
        counts = rc.read_counts(stream)
        rc.set_stats(0)
        hdr = vw.read_counters(stream)["hdr"]
        steps_per_solve = int(counts[32:32 + p.cascades].sum())
        at_cap = int(counts[64:64 + p.cascades].sum())
        # launch shapes for this workload from the library's autotuner (results do not depend on them)
        from rtgi import autotune
        if args.tuning:   # fixed launch shapes (profiling runs), else the autotuner's
            fixed = json.loads(args.tuning)
            tuned = {"rc": {k: fixed[k] for k in rc.TUNING if k in fixed},
                     "vox": {k: fixed[k] for k in ("chunk_cells", "blocks") if k in fixed}}
            rc.set_tuning(**tuned["rc"])
            vw.set_tuning(**tuned["vox"])
        else:
            tuned = autotune.Autotuner(reps=5).tune(rc, vw, stream)
        # per-pass times and the trace kernel's live duration (events between the passes)
        rc.set_timing(True)
        pass_ms = {k: [] for k in rc.PASSES}
        for _ in range(max(5, args.warmup)):
            rc.solve(vw, stream)
            for k, x in rc.pass_times().items():
                pass_ms[k].append(x)
        rc.set_timing(False)
        rc.graph_capture(vw, stream)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        for _ in range(args.warmup):
            flush.zero_()
            rc.graph_launch(stream)
        stream.synchronize()
    n_ev = args.steps
    ev_s = [torch.cuda.Event(enable_timing=True) for _ in range(n_ev)]
    ev_e = [torch.cuda.Event(enable_timing=True) for _ in range(n_ev)]
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.5)   # nvidia-smi is sampling before the timed region starts
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    unix0 = time.time()
    with torch.cuda.stream(stream):
        for k in range(n_ev):
            flush.zero_()
            ev_s[k].record(stream)
            rc.graph_launch(stream)
            ev_e[k].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    wall = time.perf_counter() - wall0
    clk = clocks.stop(unix0, unix0 + wall)
    step_ms = [a.elapsed_time(b) for a, b in zip(ev_s, ev_e)]
    total_ms = sum(step_ms)
    max_total = max_over_ranks(total_ms, dist, "cuda")
    value = whole_job_rate(n_ev, max_total / 1000.0, world)

    # end to end through the public API with host buffers: every step copies its frame + G-buffer from pinned host
    # memory and reads its irradiance back into pinned host memory; rtgi.pipeline overlaps those copies of
    # neighbouring frames with the solve (two cascade sets, upload / compute / download streams)
    depth_h = torch.from_numpy(rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).copy()).pin_memory()
    normal_h = torch.from_numpy(rc.read_buffer(_lib.GI_RC_NORMAL).view(np.uint16).copy()).pin_memory()
    frame_h = torch.from_numpy(F.copy()).pin_memory()
    # the host's normals as three halves per pixel (the path reads no alpha): 6 bytes a pixel over the bus
    normal_rgb_h = torch.from_numpy(np.ascontiguousarray(normal_h.numpy().reshape(-1, 4)[:, :3]).reshape(-1)).pin_memory()
    shadow_in = (sg, desc["shadow_map"]) if desc["shadow_map"] else None
    n_e2e = max(3, min(n_ev, 400))
    e2e_out = run_e2e(ctx, vw, p, W, H, F, (frame_h, depth_h, normal_rgb_h), shadow_in, tuned, n_e2e, dist, world)
    # the same with four halves per normal, and with the irradiance stored and read back as f32 as well
    e2e_more = {"rgba16f_normals": run_e2e(ctx, vw, p, W, H, F, (frame_h, depth_h, normal_h), shadow_in, tuned, n_e2e,
                                           dist, world),
                "three_slots": run_e2e(ctx, vw, p, W, H, F, (frame_h, depth_h, normal_rgb_h), shadow_in, tuned, n_e2e,
                                       dist, world, slots=3)}
    if p.irr16:
        e2e_more["rgba16f_normals_f32_irradiance"] = run_e2e(ctx, vw, dataclasses.replace(p, irr16=False), W, H, F,
                                                              (frame_h, depth_h, normal_h), shadow_in, tuned, n_e2e,
                                                              dist, world)

    # two frames in flight: a second voxel world and cascade set solve the same workload on a second stream, the two
    # captured solves launched side by side (what a renderer does with consecutive frames); device time of the job
    in_flight = None
    if args.in_flight:
        st2 = torch.cuda.Stream()
        vw2, rc2 = gpu.VoxWorld(sg, v), gpu.Rc(ctx, p, W, H)
        with torch.cuda.stream(st2):
            rc2.set_frame(F, st2)
            rc2.render_gbuffer(sg, st2)
            if desc["shadow_map"]:
                rc2.render_shadow(sg, desc["shadow_map"], st2)
            vw2.update(s.camera.eye)
            rc2.set_tuning(**tuned["rc"])
            vw2.set_tuning(**tuned["vox"])
            rc2.solve(vw2, st2)
            rc2.graph_capture(vw2, st2)
        torch.cuda.synchronize()
        n_f = max(3, min(n_ev, 200))
        for _ in range(3):
            rc.graph_launch(stream)
            rc2.graph_launch(st2)
        torch.cuda.synchronize()
        f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        f0.record(stream)
        st2.wait_event(f0)
        for _ in range(n_f):
            rc.graph_launch(stream)
            rc2.graph_launch(st2)
        f2.record(st2)
        stream.wait_event(f2)
        f1.record(stream)
        torch.cuda.synchronize()
        f_ms = max_over_ranks(f0.elapsed_time(f1), dist, "cuda")
        in_flight = {"frames": 2, "value": whole_job_rate(2 * n_f, f_ms / 1000.0, world), "unit": "solves/s",
                     "solves": 2 * n_f, "ms_per_solve": f_ms / (2 * n_f),
                     "mode": "two voxel worlds and cascade sets, each solve replayed from its graph on its own stream; "
                             "device time from the first launch to the last solve's end, L2 not flushed between"}
        rc2.destroy()
        vw2.destroy()

    # the same solve with multi-bounce on (bounce.ts, DEFAULT_BOUNCE; the reference renderer's default): the volume
    # traced at the start of the trace pass, its irradiance on the voxels' hits
    bounce_out = None
    if args.bounce:
        with torch.cuda.stream(stream):
            rc.set_bounce(vw)
            for _ in range(max(4, args.warmup)):
                rc.solve(vw, stream)
            rc.set_timing(True)
            b_pass = {k: [] for k in rc.PASSES}
            for _ in range(5):
                rc.solve(vw, stream)
                for k, x in rc.pass_times().items():
                    b_pass[k].append(x)
            rc.set_timing(False)
            rc.graph_capture(vw, stream)
            n_b = max(3, min(n_ev, 200))
            bs, be = ([torch.cuda.Event(enable_timing=True) for _ in range(n_b)] for _ in range(2))
            for k in range(n_b):
                flush.zero_()
                bs[k].record(stream)
                rc.graph_launch(stream)
                be[k].record(stream)
            torch.cuda.synchronize()
            b_ms = sorted(a.elapsed_time(c) for a, c in zip(bs, be))
            b_total = max_over_ranks(sum(b_ms), dist, "cuda")
            bounce_out = {"value": whole_job_rate(n_b, b_total / 1000.0, world), "unit": "solves/s", "steps": n_b,
                          "ms_per_step": b_total / n_b, "p50_ms": b_ms[n_b // 2],
                          "p99_ms": b_ms[min(n_b - 1, int(math.ceil(0.99 * n_b)) - 1)],
                          "passes_ms": {k: statistics.median(x) for k, x in b_pass.items()},
                          "volume": "32 x 16 x 32 probes 1.2 m apart, 16 rays + 6 axis rays, every 2 frames",
                          "listed_probes": int(rc.read_buffer(_lib.GI_RC_BOUNCE_LIST).view(np.uint32)[0])}
            rc.set_bounce(None)
            rc.graph_capture(vw, stream)

    # the reference renderer's default method on the same scene and clipmap: world probes
    # (world-48-voxel-rc2-vrel, docs/spec/20-renderer.md:21) with the c0 history; a frame of its own (P = 48)
    dynamic_out = run_dynamic(args, ctx, stream, flush, dist, world) if args.dynamic else None
    world_out = None
    if args.world:
        world_out = run_world(args, ctx, stream, sg, vw, s, W, H, v, desc, flush, dist, world)
        world_out["items"] = run_world_items(args, ctx, stream)

    trace_ms = statistics.mean(pass_ms["giTrace"])
    alg = trace_algorithmic_bytes(rc.layout, hdr, v)
    peak, peak_kind = measured_peak()
    achieved = alg / (trace_ms / 1000.0) / 1e9
    traffic = ncu_traffic(args.workload)
    step_sorted = sorted(step_ms)
    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": n_ev,
               "warmup": args.warmup, "ms_per_step": max_total / n_ev, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, no dataset)",
               "config": {**desc, "parallelism": f"replicas x{world} (one solve stream per GPU)",
                          "l2": "flushed between steps (256 MiB write outside the step events)",
                          "timing": "CUDA events per step on the solve stream, max over ranks",
                          "tuning": {**tuned["rc"], **tuned["vox"]}},
               "p50_ms": step_sorted[len(step_sorted) // 2],
               "p99_ms": step_sorted[min(len(step_sorted) - 1, int(math.ceil(0.99 * len(step_sorted))) - 1)],
               "dda_steps_per_solve": steps_per_solve, "dda_at_cap": at_cap,
               "dda_steps_per_s": steps_per_solve * value,
               "passes_ms": {k: statistics.median(x) for k, x in pass_ms.items()},
               "shadow_map_ms": shadow_ms,
               "bounce": bounce_out,
               "in_flight": in_flight,
               "world": world_out,
               "dynamic": dynamic_out,
               "vox_counters": {"bricks": int(min(hdr[0], v.maxBricks)), "voxels": int(hdr[1]),
                                "bricksPerLevel": [int(x) for x in hdr[8:8 + v.levels]]},
               "roofline": {"kernel": "k_trace (giTrace)", "bound": "hbm", "achieved": achieved, "peak": peak,
                            "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                            "traffic": traffic, "algorithmic_bytes": alg, "launch_ms": trace_ms},
               "e2e": e2e_out,
               "e2e_variants": e2e_more,
               "gpu_launches": n_ev * (rebuild_launches(v.levels) + 3 + p.cascades),
               "clocks": clk, "wall_s": wall}
    if args.batch > 0:
        bt = run_batched(args, ctx, stream, flush)
        if out is not None:
            out["batched"] = bt
    if args.serve_rates:
        sv = run_served(args, ctx, rank, world)
        if out is not None:
            out["served"] = sv
    if args.precision_frames > 0:
        pr = run_precision(args, ctx)
        if out is not None:
            out["precision"] = pr
    # the oracle on the host cores, rank 0 at N = 1 only
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(s, v, p, F, depth_h.numpy().reshape(H, W),
                                           normal_h.numpy().view(np.float16).reshape(H, W, 4).astype(np.float32),
                                           desc["shadow_map"])
    for h in (rc, vw, sg, ctx):
        h.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="colonnade", choices=["colonnade", "room"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--tuning", default=None, help="fixed launch shapes as JSON (skips the autotuner)")
    ap.add_argument("--no-bounce", dest="bounce", action="store_false", help="skip the multi-bounce measurement")
    ap.add_argument("--no-world", dest="world", action="store_false", help="skip the world-probe measurement")
    ap.add_argument("--no-dynamic", dest="dynamic", action="store_false",
                    help="skip the dynamic-layer measurement (64 moving boxes splatted into the layer)")
    ap.add_argument("--no-in-flight", dest="in_flight", action="store_false",
                    help="skip the two-frames-in-flight measurement")
    ap.add_argument("--batch", type=int, default=64, help="uneven solves of the batched measurement (0: skip)")
    ap.add_argument("--serve-rates", type=float, nargs="*", default=[100, 500, 1000, 2000, 5000],
                    help="request rates of the serving measurement (none: skip)")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-max", type=int, default=2000)
    ap.add_argument("--precision-frames", type=int, default=100,
                    help="frames of the atlas precision study (colonnade + 64 moving boxes; 0: skip)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
