"""Request routing for serving on several GPUs (rtgi/route.py): the placement of scenes on ranks, and the routed
serving loop as world_size-2 gloo ranks on the CPU, each with the simulated executor and clock of the scheduler
tests: every request is served exactly once, on an owner of its scene, and no rank loads a scene it does not own."""
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from rtgi import route, scenes, serve

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_place_splits_a_hot_scene_and_balances_the_rest():
    owners = route.place([5.0, 1.0, 1.0, 1.0], 2)
    assert owners[0] == [0, 1]                       # above the fair share of 4: on both ranks
    assert all(len(o) == 1 for o in owners[1:])
    held = [0.0, 0.0]
    for x, o in zip([5.0, 1.0, 1.0, 1.0], owners):
        for r in o:
            held[r] += x / len(o)
    assert held == [4.5, 3.5]                        # 2.5 + 1 + 1 and 2.5 + 1


def test_place_properties():
    rng = np.random.default_rng(3)
    for trial in range(200):
        n, ranks = int(rng.integers(1, 30)), int(rng.integers(1, 9))
        loads = list(rng.lognormal(0.0, 1.0, n))
        owners = route.place(loads, ranks)
        fair = sum(loads) / ranks
        held = [0.0] * ranks
        biggest = 0.0
        for x, o in zip(loads, owners):
            assert 1 <= len(o) <= ranks and len(set(o)) == len(o) and all(0 <= r < ranks for r in o)
            assert len(o) == min(ranks, max(1, int(np.ceil(x / fair - 1e-9))))
            for r in o:
                held[r] += x / len(o)
            biggest = max(biggest, x / len(o))
        assert max(held) <= fair + biggest + 1e-9   # list scheduling bound
        assert route.place(loads, ranks) == owners    # deterministic: every rank derives the same table


def test_requests_go_to_owners_and_alternate_on_replicas():
    owners = [[0, 1], [1], [0]]
    reqs = serve.poisson_arrivals(1000.0, 300, 3, seed=4)
    parts = [route.share(reqs, owners, r) for r in (0, 1)]
    assert sorted(q.rid for p in parts for q in p) == list(range(300))
    for r, part in enumerate(parts):
        assert all(r in owners[q.scene] for q in part)
        assert [q.arrival for q in part] == sorted(q.arrival for q in part)
    hot = [q for q in reqs if q.scene == 0]
    assert {route.owner(owners, q) for q in hot} == {0, 1}


def test_single_rank_is_the_plain_server():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_serve import FakeClock, FakeExecutor
    specs = [scenes.batch_spec(1000 + s) for s in range(6)]
    clock = FakeClock()
    ex = FakeExecutor(clock)
    rs = route.RoutedServer(lambda mine: serve.Server(ex, specs, slots=4, hbm_budget=1e9), specs, 0, 1)
    assert rs.mine == list(range(6))
    st = rs.run(serve.poisson_arrivals(800.0, 120, len(specs), seed=2), clock)
    assert st["completed"] == 120 and st["ranks"] == 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "real-time-gi-lab_b200")]
    import datetime
    import torch.distributed as dist
    from rtgi import route, scenes, serve
    from test_serve import FakeClock, FakeExecutor
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    specs = [scenes.batch_spec(1000 + s) for s in range(12)]
    clock = FakeClock()
    ex = FakeExecutor(clock)
    rs = route.RoutedServer(lambda mine: serve.Server(ex, specs, slots=4, hbm_budget=4 * ex.cost), specs, rank, world)
    reqs = serve.poisson_arrivals(3000.0, 400, len(specs), seed=5)
    st = rs.run(reqs, clock)
    loaded = sorted({sid for op, sid in ex.log if op == "load"})
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"stats": st, "mine": rs.mine, "owners": rs.owners, "loaded": loaded}, f)


def test_two_gloo_ranks_route_every_request_once(tmp_path):
    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert res[0]["owners"] == res[1]["owners"]
    assert res[0]["stats"] == res[1]["stats"]                  # the pooled statistics, the same on every rank
    st = res[0]["stats"]
    assert st["completed"] == 400 and st["ranks"] == 2
    assert sum(p["completed"] for p in st["per_rank"]) == 400
    assert all(p["completed"] > 0 for p in st["per_rank"])
    for r in res:                                              # only owned scenes are loaded (HBM budget: 4 scenes)
        assert set(r["loaded"]) <= set(r["mine"])
    assert set(res[0]["mine"]) | set(res[1]["mine"]) == set(range(12))
