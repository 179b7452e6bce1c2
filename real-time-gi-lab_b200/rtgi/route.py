"""Request routing for the serving loop on several GPUs, one process per GPU (no counterpart in the reference, which
renders on one device).

Placement: every scene is owned by one rank, or by several when its expected load is above one rank's fair share.
Owners are picked longest-processing-time first: the scenes' pieces (a scene of expected load x split into
ceil(x / fair) equal pieces, fair = total / ranks) in decreasing load, each to the least-loaded rank that does not hold
the scene yet.  A scene's clipmap, atlases and captured frame graph live only on its owners; each rank runs its own
`serve.Server` (continuous batching, HBM budget) over the requests routed to it.

Routing: request r goes to owners[r.scene][r.rid mod len(owners)]: a scene with one owner always to that rank, a
replicated one alternating among its owners.  Every rank derives the same table from the same scene specs and filters
the same arrival stream with it, so requests need no exchange on the data path; the ranks exchange only their results
at the end (`all_gather_object` over the process group)."""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence

from .serve import Request, summarize


def solve_cost(spec: dict) -> float:
    """Expected device time of one request (ms), a linear proxy: the rebuild grows with the triangles, the cascades
    with the pixels (0.19 ms for 262k triangles and 0.33 ms for 1920x1080 in the colonnade solve)."""
    return 0.01 + 0.73e-6 * spec["tris"] + 0.16e-6 * spec["width"] * spec["height"]


def place(loads: Sequence[float], ranks: int) -> List[List[int]]:
    """Owners per scene (ranks in increasing order) for the scenes' expected loads (request share x solve cost)."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    if any(x < 0 or not math.isfinite(x) for x in loads):
        raise ValueError("loads must be finite and >= 0")
    total = float(sum(loads))
    fair = total / ranks if total > 0 else 1.0
    pieces = []
    for sid, x in enumerate(loads):
        k = min(ranks, max(1, math.ceil(x / fair - 1e-9)))
        pieces += [(x / k, sid)] * k
    pieces.sort(key=lambda p: (-p[0], p[1]))
    held = [0.0] * ranks
    owners: List[List[int]] = [[] for _ in loads]
    for x, sid in pieces:
        r = min((r for r in range(ranks) if r not in owners[sid]), key=lambda r: (held[r], r))
        owners[sid].append(r)
        held[r] += x
    return [sorted(o) for o in owners]


def owner(owners: List[List[int]], rq: Request) -> int:
    o = owners[rq.scene]
    return o[rq.rid % len(o)]


def share(requests: Sequence[Request], owners: List[List[int]], rank: int) -> List[Request]:
    """This rank's requests, in arrival order."""
    return [rq for rq in requests if owner(owners, rq) == rank]


def pooled(done: List[Request], extra: dict) -> dict:
    """Statistics over the requests of every rank (arrival times share the ranks' common stream clock)."""
    return summarize(done, extra)


class RoutedServer:
    """One rank's part of the routed serving loop.  make_server(scene_ids) builds this rank's Server over its own
    executor; only the scenes this rank owns are ever loaded there."""

    def __init__(self, make_server: Callable, specs: List[dict], rank: int, world: int, group=None,
                 loads: Optional[Sequence[float]] = None):
        self.specs, self.rank, self.world, self.group = specs, rank, world, group
        self.owners = place(loads if loads is not None else [solve_cost(s) for s in specs], world)
        self.mine = [sid for sid, o in enumerate(self.owners) if rank in o]
        self.server = make_server(self.mine)

    def run(self, requests: List[Request], clock=None) -> dict:
        """Serves this rank's share; returns the pooled statistics of every rank (the same dict on every rank)."""
        return self.run_with(self.server.run, requests, clock)

    def run_with(self, serve_fn: Callable, requests: List[Request], clock=None) -> dict:
        """The same with another loop over this rank's share: serve_fn(requests, clock) -> statistics (the plain
        one-at-a-time loop, routed the same way, for comparison)."""
        mine = share(requests, self.owners, self.rank)
        self._barrier()   # the ranks' stream clocks start together
        local = serve_fn(mine, clock) if mine else {"completed": 0}
        rows = [(rq.rid, rq.scene, rq.arrival, rq.start, rq.done) for rq in mine]
        everything = self._gather((self.rank, rows, local))
        done, per_rank = [], {}
        for rank, rs, st in everything:
            per_rank[rank] = st
            for rid, scene, arrival, start, fin in rs:
                r = Request(rid, scene, 0.0, arrival)
                r.start, r.done = start, fin
                done.append(r)
        if len(done) != len(requests) or len({r.rid for r in done}) != len(requests):
            raise RuntimeError(f"routing lost or repeated requests: {len(done)} served of {len(requests)}")
        return pooled(done, {"ranks": self.world, "per_rank": [per_rank[r] for r in range(self.world)]})

    def _barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier(group=self.group)

    def _gather(self, item) -> list:
        if self.world == 1:
            return [item]
        import torch.distributed as dist
        out = [None] * self.world
        dist.all_gather_object(out, item, group=self.group)
        return out
