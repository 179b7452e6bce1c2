"""bench.py's N > 1 host logic (replicas: rendezvous, barrier, max over ranks, whole-job rate, rank-0-only reference
arm) with world_size-2 gloo ranks on the CPU."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_ranks(world, backend="gloo", timeout_s=60)
    dist.barrier()
    local_ms = 10.0 * (rank + 1)                # rank 1 is the slower replica
    mx = bench.max_over_ranks(local_ms, dist, "cpu")
    rate = bench.whole_job_rate(100, mx / 1000.0, world)
    ref = bench.run_reference(None, rank) if rank != 0 else "skipped"   # other ranks exit without work
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"max": mx, "rate": rate, "ref": ref}, f)


def test_two_gloo_ranks(tmp_path):
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    for r in res:
        assert r["max"] == 20.0                   # every rank sees the slowest rank's time
        assert r["rate"] == pytest.approx(2 * 100 / 0.020)
    assert res[1]["ref"] is None


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_ranks(1) is None
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(10, 2.0, 1) == 5.0
