"""Worlds: instances of a scene's static part, its triangles grouped into chunks, and the clustered (LOD) copies the
voxel build reads when a chunk's finest window is a coarse level (src/core/world.ts withWorld / selectItems, and the
per-frame windows of voxel.ts:868-885).  Host-side, f64 like the reference's numbers; the clustered vertices are
rounded to f32 where the reference stores them into its Float32Arrays.

The voxel build then reads a per-frame list of work items (instance, chunk rows, first level) instead of every
triangle (gi_vox_set_world / gi_vox_set_items); a triangle's key is instance * rows + row, and instance i moves its
triangles by its offset.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import mathx

CHUNK = 8                 # chunk cells (m), world.ts:21
DEFAULT_LOD0_CELL = 0.1   # world.ts:24
LOD0_KEEP = 0.5           # world.ts:28
MOTION_MARGIN = 0.15      # world.ts:30
MAX_INSTANCES = 1024   # voxel.ts:742
MAX_ITEMS = 16384       # voxel.ts:742


@dataclass
class WorldChunk:
    lo: Tuple[float, float, float]
    hi: Tuple[float, float, float]
    full: np.ndarray                     # table rows of the chunk, ascending
    lod: List[np.ndarray]                # per start level s: the rows voxelised from level s on


@dataclass
class World:
    instances: List[Tuple[float, float, float]]
    static_triangles: int
    static_vertices: int
    v0: float
    levels: int
    chunks: List[WorldChunk]
    lod_first_vertex: int
    lod_vertex_count: int
    lod_table: np.ndarray                # (n, 4) rows of the clustered triangles, after the scene's rows
    rows: int = 0                        # the key stride: the scene's rows + the clustered rows
    list_off: List[List[int]] = field(default_factory=list)   # per chunk and level: offset of its rows in lists()

    def lists(self) -> np.ndarray:
        """Every chunk's row lists, chunk by chunk, level by level (the offsets are list_off)."""
        parts = [l for ch in self.chunks for l in ch.lod]
        return np.concatenate(parts).astype(np.uint32) if parts else np.zeros(0, np.uint32)


def _dir_key(x: float, y: float, z: float) -> int:
    """world.ts:57-61: the dominant axis of a normal and its sign, 0..5."""
    ax, ay, az = abs(x), abs(y), abs(z)
    if ax >= ay and ax >= az:
        return 0 if x >= 0 else 1
    if ay >= az:
        return 2 if y >= 0 else 3
    return 4 if z >= 0 else 5


def _js_num(x: float) -> str:
    """A JS number as String() prints an integral value (the chunk and cluster keys are integers)."""
    return str(int(x)) if x == int(x) else repr(x)


def with_world(scene, instances: Sequence[Sequence[float]], v0: float, levels: int, lod0_cell: float = 0.0):
    """withWorld (world.ts:64-172) for a scene whose every triangle is static.  Returns (scene', world): scene' has the
    clustered vertices appended (not drawn) and its triangle table grown by the clustered rows."""
    import dataclasses
    inst = [tuple(float(a) for a in o) for o in instances]
    if not inst or any(x != 0 for x in inst[0]):
        raise ValueError("instance 0 must be at the origin")
    if len(inst) > MAX_INSTANCES:
        raise ValueError("too many instances")
    P = np.asarray(scene.positions, np.float32).astype(np.float64).reshape(-1)
    N = np.asarray(scene.normals, np.float32).astype(np.float64).reshape(-1)
    table = np.asarray(scene.tri, np.uint32).reshape(-1)
    T = int(scene.tri.shape[0])
    V0 = P.size // 3
    by_chunk: Dict[str, List[int]] = {}
    for t in range(T):
        c = [0.0, 0.0, 0.0]
        for q in range(3):
            v = int(table[t * 4 + q])
            for a in range(3):
                c[a] += P[v * 3 + a] / 3
        k = ",".join(_js_num(math.floor(x / CHUNK)) for x in c)
        by_chunk.setdefault(k, []).append(t)
    keys = sorted(by_chunk)
    lod_pos: List[float] = []
    lod_nrm: List[float] = []
    lod_uv: List[int] = []        # per cluster vertex the source vertex of its uv
    lod_rows: List[int] = []
    first_row = T
    pending: List[list] = [[] for _ in range(levels)]
    chunks: List[WorldChunk] = []
    for ci, k in enumerate(keys):
        tris = by_chunk[k]
        lo = [math.inf] * 3
        hi = [-math.inf] * 3
        for t in tris:
            for q in range(3):
                v = int(table[t * 4 + q])
                for a in range(3):
                    x = P[v * 3 + a]
                    lo[a] = min(lo[a], x)
                    hi[a] = max(hi[a], x)
        full = np.asarray(tris, np.uint32)
        lod: List[np.ndarray] = []
        for s in range(levels):
            cell = lod0_cell if s == 0 else v0 * 2 ** (s - 1)
            if cell == 0:
                lod.append(full)
                continue
            clusters: Dict[str, dict] = {}
            tri_cl = []
            for t in tris:
                m = int(table[t * 4 + 3])
                ids = []
                for q in range(3):
                    v = int(table[t * 4 + q])
                    d = _dir_key(N[v * 3], N[v * 3 + 1], N[v * 3 + 2]) if s == 0 else 0
                    ck = f"{m}|{d}|" + ",".join(_js_num(math.floor(P[v * 3 + a] / cell)) for a in range(3))
                    cl = clusters.get(ck)
                    if cl is None:
                        cl = clusters[ck] = {"id": len(clusters), "sum": [0.0, 0.0, 0.0], "n": 0, "nrm": [0.0, 0.0, 0.0],
                                             "verts": []}
                    if v not in cl["verts"]:
                        cl["verts"].append(v)
                        cl["n"] += 1
                        for a in range(3):
                            cl["sum"][a] += P[v * 3 + a]
                            cl["nrm"][a] += N[v * 3 + a]
                    ids.append(cl["id"])
                tri_cl.append(ids)
            vbase = V0 + len(lod_pos) // 3
            for cl in sorted(clusters.values(), key=lambda c: c["id"]):
                p = [x / cl["n"] for x in cl["sum"]]
                l = mathx.hypot(*cl["nrm"])
                best, bd = cl["verts"][0], math.inf
                for v in cl["verts"]:
                    dd = (P[v * 3] - p[0]) ** 2 + (P[v * 3 + 1] - p[1]) ** 2 + (P[v * 3 + 2] - p[2]) ** 2
                    if dd < bd:
                        bd, best = dd, v
                lod_pos.extend(p)
                lod_nrm.extend([x / l for x in cl["nrm"]] if l > 1e-12 else [N[best * 3], N[best * 3 + 1], N[best * 3 + 2]])
                lod_uv.append(best)   # the cluster's uv: the vertex nearest the mean's (world.ts:124, 137)
            seen = set()
            mine = []
            for i, t in enumerate(tris):
                m = int(table[t * 4 + 3])
                ids = tri_cl[i]
                k2 = f"{m}|" + ",".join(str(x) for x in sorted(ids))
                if k2 in seen:
                    continue
                seen.add(k2)
                collapsed = ids[0] == ids[1] or ids[1] == ids[2] or ids[0] == ids[2]
                mine.append((ci, t, collapsed, [vbase + ids[0], vbase + ids[1], vbase + ids[2]], m))
            if s == 0 and len(mine) > LOD0_KEEP * len(tris):
                lod.append(full)
                continue
            pending[s].extend(mine)
            lod.append(np.zeros(0, np.uint32))
        chunks.append(WorldChunk(tuple(x - MOTION_MARGIN for x in lo), tuple(x + MOTION_MARGIN for x in hi), full, lod))
    for s, lst in enumerate(pending):
        if not lst:
            continue
        lst.sort(key=lambda e: (-int(e[2]), e[1]))
        per_chunk: Dict[int, List[int]] = {}
        for ci, t, collapsed, vv, m in lst:
            per_chunk.setdefault(ci, []).append(first_row + len(lod_rows) // 4)
            lod_rows.extend([vv[0], vv[1], vv[2], m])
        for ci, rows in per_chunk.items():
            chunks[ci].lod[s] = np.asarray(rows, np.uint32)
    nv = len(lod_pos) // 3
    pos = np.concatenate([np.asarray(scene.positions, np.float32).reshape(-1, 3),
                          np.asarray(lod_pos, np.float64).reshape(-1, 3).astype(np.float32)])
    nrm = np.concatenate([np.asarray(scene.normals, np.float32).reshape(-1, 3),
                          np.asarray(lod_nrm, np.float64).reshape(-1, 3).astype(np.float32)])
    lod_table = np.asarray(lod_rows, np.uint32).reshape(-1, 4)
    tri = np.concatenate([np.asarray(scene.tri, np.uint32).reshape(-1, 4), lod_table])
    extra = {}
    if getattr(scene, "uvs", None) is not None:
        uv0 = np.asarray(scene.uvs, np.float32).reshape(-1, 2)
        extra["uvs"] = np.concatenate([uv0, uv0[np.asarray(lod_uv, np.int64)].reshape(-1, 2)]).astype(np.float32)
    out = dataclasses.replace(scene, positions=pos, normals=nrm, tri=tri, **extra)
    world = World(inst, T, V0, v0, levels, chunks, V0, nv, lod_table, rows=int(tri.shape[0]))
    off = 0
    for ch in chunks:
        row = []
        for l in ch.lod:
            row.append(off)
            off += len(l)
        world.list_off.append(row)
    return out, world


def windows(v0: float, levels: int, G: int, eye: Sequence[float]) -> List[Tuple[tuple, tuple]]:
    """The clipmap windows per level in metres, [lo, hi) (writeUniform, voxel.ts:871-876; f64)."""
    out = []
    for L in range(levels):
        bs = v0 * 2 ** L * 8
        o = [math.floor(eye[a] / bs) - G / 2 for a in range(3)]
        out.append((tuple(x * bs for x in o), tuple((x + G) * bs for x in o)))
    return out


@dataclass
class WorkItem:
    inst: int
    start: int
    list: int
    first: int
    count: int


def select_items(world: World, wins) -> List[WorkItem]:
    """selectItems (world.ts:179-199): the chunks of the instances inside the windows, from their finest window on, in
    (instance, chunk) order."""
    items = []
    for inst, o in enumerate(world.instances):
        for c, ch in enumerate(world.chunks):
            s = -1
            for L, (wlo, whi) in enumerate(wins):
                if all(ch.lo[a] + o[a] < whi[a] and ch.hi[a] + o[a] > wlo[a] for a in range(3)):
                    s = L
                    break
            if s < 0:
                continue
            n = len(ch.lod[s])
            if n > 0:
                items.append(WorkItem(inst, s, world.list_off[c][s], 0, n))
    if len(items) > MAX_ITEMS:
        raise ValueError(f"too many work items: {len(items)}")
    return items


def item_records(items: List[WorkItem]) -> Tuple[np.ndarray, int]:
    """The items as the build reads them (voxel.ts:883-885): (first thread, source, instance, first level) each, the
    source an offset into the row lists, or 0x80000000 | first row for a contiguous range; and the thread count."""
    rec = np.zeros((len(items), 4), np.uint32)
    threads = 0
    for k, it in enumerate(items):
        rec[k] = (threads, (0x80000000 | it.first) if it.list < 0 else it.list, it.inst, it.start)
        threads += it.count
    return rec, threads
