"""Scene data for the GI path (src/core/gltf.ts SceneData, src/core/scenes.ts Builder and leakRoom) and the seeded
procedural scenes the benchmarks run on.

A ``Scene`` holds what the voxel build and the G-buffer read: f32 positions and normals, the triangle table
(absolute vertex indices + material, voxel.ts:730-739 triangleTable) in the reference's order (the triangles of
material 0 first, as Builder.scene() emits one primitive per material), and the materials.  The reference's
materials carry no emission; ``Material.emissive`` is this build's addition (radiance added at a voxel hit).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import mathx
from .frame import Camera

MATERIAL_DTYPE = np.dtype([("base_color", "<f4", (4,)), ("flags", "<u4"), ("alpha_cutoff", "<f4"),
                           ("emissive", "<f4", (3,)), ("base_color_tex", "<u4"), ("reserved", "<u4", (2,))])
assert MATERIAL_DTYPE.itemsize == 48

FLAG_ALPHA_MASK, FLAG_DOUBLE_SIDED, FLAG_TOON, FLAG_OBJECT = 1, 2, 4, 8


@dataclass
class Material:
    name: str
    base_color: tuple = (0.7, 0.7, 0.7, 1.0)
    flags: int = 0
    alpha_cutoff: float = 0.5
    emissive: tuple = (0.0, 0.0, 0.0)
    base_color_tex: int = 0        # 1 + the scene's texture layer (layers.x of the reference); 0: untextured


GREY = Material("grey", (0.7, 0.7, 0.7, 1.0))   # scenes.ts:173


@dataclass
class Scene:
    name: str
    positions: np.ndarray          # (V, 3) f32
    normals: np.ndarray            # (V, 3) f32
    tri: np.ndarray                # (T, 4) u32: i0, i1, i2, material
    materials: List[Material]
    camera: Camera
    sun_dir: tuple = (0.0, 1.0, 0.0)
    sun_e: tuple = (0.0, 0.0, 0.0)
    sky: tuple = (0.0, 0.0, 0.0)
    uvs: Optional[np.ndarray] = None        # (V, 2) f32 texture coordinates, or None
    textures: Optional[np.ndarray] = None   # (layers, size, size, 4) u8 base colour images (sRGB rgb, linear alpha)

    @property
    def triangle_count(self) -> int:
        return int(self.tri.shape[0])

    def material_array(self) -> np.ndarray:
        a = np.zeros(len(self.materials), dtype=MATERIAL_DTYPE)
        for i, m in enumerate(self.materials):
            a[i]["base_color"] = m.base_color
            a[i]["flags"] = m.flags
            a[i]["alpha_cutoff"] = m.alpha_cutoff
            a[i]["emissive"] = m.emissive
            a[i]["base_color_tex"] = m.base_color_tex
        return a


class Builder:
    """Builder (scenes.ts:176-211): quads of 4 new vertices with the face normal, boxes with outward faces."""

    def __init__(self, materials: Optional[List[Material]] = None):
        self.materials = list(materials) if materials else [GREY]
        self.pos: List[float] = []
        self.nrm: List[float] = []
        self.idx: List[List[int]] = [[] for _ in self.materials]
        self.mat = 0
        self.offset = [0.0, 0.0, 0.0]
        self._extra_pos: List[np.ndarray] = []

    def quad(self, a, b, c, d):
        e1 = [b[0] - a[0], b[1] - a[1], b[2] - a[2]]
        e2 = [c[0] - a[0], c[1] - a[1], c[2] - a[2]]
        n = mathx.normalize([e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]])
        base = len(self.pos) // 3
        for p in (a, b, c, d):
            self.pos += [p[0] + self.offset[0], p[1] + self.offset[1], p[2] + self.offset[2]]
            self.nrm += n
        self.idx[self.mat] += [base, base + 1, base + 2, base, base + 2, base + 3]

    def quad_facing(self, a, b, c, d, want):
        """quad() with the corner order flipped when its face normal points away from ``want``."""
        e1 = [b[i] - a[i] for i in range(3)]
        e2 = [c[i] - a[i] for i in range(3)]
        n = [e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]]
        if n[0] * want[0] + n[1] * want[1] + n[2] * want[2] < 0:
            a, b, c, d = a, d, c, b
        self.quad(a, b, c, d)

    def box(self, c, h):
        x0, y0, z0 = c[0] - h[0], c[1] - h[1], c[2] - h[2]
        x1, y1, z1 = c[0] + h[0], c[1] + h[1], c[2] + h[2]
        self.quad([x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1])
        self.quad([x1, y0, z0], [x0, y0, z0], [x0, y1, z0], [x1, y1, z0])
        self.quad([x0, y0, z0], [x0, y0, z1], [x0, y1, z1], [x0, y1, z0])
        self.quad([x1, y0, z1], [x1, y0, z0], [x1, y1, z0], [x1, y1, z1])
        self.quad([x0, y1, z1], [x1, y1, z1], [x1, y1, z0], [x0, y1, z0])
        self.quad([x0, y0, z0], [x1, y0, z0], [x1, y0, z1], [x0, y0, z1])

    def mesh(self, pos: np.ndarray, nrm: np.ndarray, tris: np.ndarray):
        """Appends an indexed mesh (f64 positions/normals, local triangle indices) to the current material."""
        base = len(self.pos) // 3
        self.pos += (pos + np.asarray(self.offset)).reshape(-1).tolist()
        self.nrm += nrm.reshape(-1).tolist()
        self.idx[self.mat] += (tris.reshape(-1) + base).tolist()

    def scene(self, name: str, camera: Camera, **kw) -> Scene:
        positions = np.asarray(self.pos, dtype=np.float64).astype(np.float32).reshape(-1, 3)
        normals = np.asarray(self.nrm, dtype=np.float64).astype(np.float32).reshape(-1, 3)
        rows = []
        for m, l in enumerate(self.idx):
            if not l:
                continue
            a = np.asarray(l, dtype=np.uint32).reshape(-1, 3)
            rows.append(np.concatenate([a, np.full((a.shape[0], 1), m, dtype=np.uint32)], axis=1))
        tri = np.concatenate(rows, axis=0) if rows else np.zeros((0, 4), dtype=np.uint32)
        return Scene(name, positions, normals, np.ascontiguousarray(tri), list(self.materials), camera, **kw)


def leak_room(t: float) -> Scene:
    """leakRoom (scenes.ts:261-278): a closed room on a floor of 24 x 24 cells, walls and roof t thick."""
    b = Builder()
    cells, size = 24, 8
    step = size / cells
    for z in range(cells):
        for x in range(cells):
            x0, z0 = -size / 2 + 1.5 + x * step, -size / 2 + z * step
            b.quad([x0, 0, z0 + step], [x0 + step, 0, z0 + step], [x0 + step, 0, z0], [x0, 0, z0])
    W, H, D = 3, 2.7, 2.25
    b.box([-t / 2, H / 2, 0], [t / 2, H / 2, D + t])
    b.box([W + t / 2, H / 2, 0], [t / 2, H / 2, D + t])
    b.box([W / 2, H / 2, -D - t / 2], [W / 2, H / 2, t / 2])
    b.box([W / 2, H / 2, D + t / 2], [W / 2, H / 2, t / 2])
    b.box([W / 2, H + t / 2, 0], [W / 2 + t, t / 2, D + t])
    return b.scene(f"leak-{t:g}", Camera((2.6, 1.6, 1.8), (0.2, 1.0, -1.4), 75, 0.05), sun_dir=(-1, 1.1, 0.35))


class PCG32:
    """PCG32 (O'Neill 2014, pcg32_srandom / pcg32_random): the seeded stream of the procedural scenes."""
    MULT = 6364136223846793005
    MASK = (1 << 64) - 1

    def __init__(self, seed: int, stream: int = 54):
        self.state = 0
        self.inc = ((stream << 1) | 1) & self.MASK
        self.next_u32()
        self.state = (self.state + seed) & self.MASK
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * self.MULT + self.inc) & self.MASK
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u32() >> 8) * (1.0 / 16777216.0))


def room_scene(seed: int = 0, n_boxes: int = 200) -> Scene:
    """Small procedural scene: a 10 x 10 x 4 m room (12 inward triangles), axis-aligned boxes with centres uniform in
    the room, sides uniform 0.2-1.5 m, albedo uniform 0.1-0.9 per channel, and one 1 x 1 m emissive quad of radiance 10
    under the ceiling.  The camera stands in the room; boxes that would hold it are drawn again."""
    rng = PCG32(seed)
    eye = (5.5, 1.7, 5.5)
    mats = [Material("room", (0.75, 0.75, 0.75, 1.0)), Material("lamp", (0.9, 0.9, 0.9, 1.0), emissive=(10.0, 10.0, 10.0))]
    boxes = []
    while len(boxes) < n_boxes:
        c = [rng.uniform(0, 10), rng.uniform(0, 4), rng.uniform(0, 10)]
        h = [rng.uniform(0.2, 1.5) / 2, rng.uniform(0.2, 1.5) / 2, rng.uniform(0.2, 1.5) / 2]
        alb = (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), 1.0)
        if all(abs(eye[a] - c[a]) < h[a] + 0.3 for a in range(3)):
            continue
        boxes.append((c, h, alb))
    for i, (_, _, alb) in enumerate(boxes):
        mats.append(Material(f"box{i}", alb))
    b = Builder(mats)
    b.mat = 0   # the room, faces inward
    X, Y, Z = 10.0, 4.0, 10.0
    b.quad_facing([0, 0, 0], [X, 0, 0], [X, 0, Z], [0, 0, Z], (0, 1, 0))      # floor
    b.quad_facing([0, Y, Z], [X, Y, Z], [X, Y, 0], [0, Y, 0], (0, -1, 0))     # ceiling
    b.quad_facing([0, 0, 0], [0, Y, 0], [X, Y, 0], [X, 0, 0], (0, 0, 1))      # z = 0 wall
    b.quad_facing([X, 0, Z], [X, Y, Z], [0, Y, Z], [0, 0, Z], (0, 0, -1))     # z = Z wall
    b.quad_facing([0, 0, Z], [0, Y, Z], [0, Y, 0], [0, 0, 0], (1, 0, 0))      # x = 0 wall
    b.quad_facing([X, 0, 0], [X, Y, 0], [X, Y, Z], [X, 0, Z], (-1, 0, 0))     # x = X wall
    b.mat = 1
    b.quad_facing([4.5, 3.95, 5.5], [5.5, 3.95, 5.5], [5.5, 3.95, 4.5], [4.5, 3.95, 4.5], (0, -1, 0))   # lamp
    for i, (c, h, _) in enumerate(boxes):
        b.mat = 2 + i
        b.box(c, h)
    return b.scene(f"room-{seed}", Camera(eye, (1.0, 1.0, 1.5), 60, 0.05), sun_dir=(0.3, 1.0, 0.2))


def _cylinder(cx: float, cz: float, r: float, h: float, seg: int, rings: int):
    """Smooth cylinder side about the y axis: (seg + 1) x (rings + 1) vertices with radial normals, 2 seg rings
    triangles wound counter-clockwise seen from outside."""
    u = np.arange(seg + 1) / seg * 2 * math.pi
    v = np.arange(rings + 1) / rings * h
    cu, su = np.cos(u), np.sin(u)
    pos = np.stack([np.broadcast_to(cx + r * cu, (rings + 1, seg + 1)), np.broadcast_to(v[:, None], (rings + 1, seg + 1)),
                    np.broadcast_to(cz + r * su, (rings + 1, seg + 1))], axis=-1).reshape(-1, 3)
    nrm = np.stack([np.broadcast_to(cu, (rings + 1, seg + 1)), np.zeros((rings + 1, seg + 1)),
                    np.broadcast_to(su, (rings + 1, seg + 1))], axis=-1).reshape(-1, 3)
    j, i = np.meshgrid(np.arange(rings), np.arange(seg), indexing="ij")
    a = (j * (seg + 1) + i).reshape(-1)
    b_ = a + 1
    c = a + (seg + 1)
    d = c + 1
    # outward: (a, c, d) and (a, d, b) are counter-clockwise seen from outside for u increasing towards +z
    tris = np.concatenate([np.stack([a, c, d], 1), np.stack([a, d, b_], 1)], axis=0)
    return pos, nrm, tris


def colonnade_scene(seed: int = 0, nx: int = 40, nz: int = 16, rings: int = 8, seg: int = 24) -> Scene:
    """Large procedural scene (~260k triangles): an nx x nz grid of columns 2.5 m apart (seg-segment cylinders of
    radius 0.3 m and height 8 m, rings bands high), box beams joining neighbouring column heads, a tiled floor, four
    perimeter walls, four 2 x 2 m emissive panels (radiance ~10) under the beams, and a directional sun."""
    rng = PCG32(seed, stream=7)
    mats = [Material("floor", (0.6, 0.55, 0.5, 1.0)), Material("stone", (0.8, 0.78, 0.72, 1.0)),
            Material("beam", (0.7, 0.5, 0.35, 1.0)), Material("wall", (0.5, 0.55, 0.6, 1.0))]
    lamp_cols = [(10.0, 9.5, 8.5), (8.5, 9.5, 10.0), (10.0, 8.0, 7.0), (9.0, 10.0, 9.0)]
    for k, e in enumerate(lamp_cols):
        mats.append(Material(f"lamp{k}", (0.9, 0.9, 0.9, 1.0), emissive=e))
    b = Builder(mats)
    sp = 2.5
    x0, z0 = -(nx - 1) * sp / 2, -(nz - 1) * sp / 2
    xs = [x0 + i * sp for i in range(nx)]
    zs = [z0 + j * sp for j in range(nz)]
    b.mat = 0
    for j in range(nz):
        for i in range(nx):
            ax, az = xs[i] - sp / 2, zs[j] - sp / 2
            b.quad([ax, 0, az + sp], [ax + sp, 0, az + sp], [ax + sp, 0, az], [ax, 0, az])
    b.mat = 1
    for j in range(nz):
        for i in range(nx):
            pos, nrm, tris = _cylinder(xs[i], zs[j], 0.3, 8.0, seg, rings)
            b.mesh(pos, nrm, tris)
    b.mat = 2
    for j in range(nz):
        for i in range(nx - 1):
            b.box([xs[i] + sp / 2, 8.25, zs[j]], [sp / 2, 0.25, 0.3])
    for j in range(nz - 1):
        for i in range(nx):
            b.box([xs[i], 8.25, zs[j] + sp / 2], [0.3, 0.25, sp / 2])
    b.mat = 3
    hx, hz = nx * sp / 2, nz * sp / 2
    b.box([0, 5, -hz - 0.15], [hx + 0.3, 5, 0.15])
    b.box([0, 5, hz + 0.15], [hx + 0.3, 5, 0.15])
    b.box([-hx - 0.15, 5, 0], [0.15, 5, hz])
    b.box([hx + 0.15, 5, 0], [0.15, 5, hz])
    for k in range(4):
        b.mat = 4 + k
        cx = xs[int(rng.uniform(2, nx - 3))] + sp / 2
        cz = zs[int(rng.uniform(2, nz - 3))] + sp / 2
        b.quad_facing([cx - 1, 7.5, cz + 1], [cx + 1, 7.5, cz + 1], [cx + 1, 7.5, cz - 1], [cx - 1, 7.5, cz - 1], (0, -1, 0))
    # the eye stands in the aisle between four columns (columns stand at odd multiples of 1.25 m)
    cam = Camera((0.0, 1.7, 0.0), (21.25, 1.3, -3.75), 60, 0.05)
    from .frame import SUN_E, SKY
    return b.scene(f"colonnade-{seed}", cam, sun_dir=(-0.4, 1.0, 0.3), sun_e=SUN_E, sky=SKY)


def mixed_scene(seed: int, target_tris: int, area: float = 40.0, name: str = "") -> Scene:
    """Procedural box/column mix of about target_tris triangles: a tiled ground, columns (16-segment cylinders) for
    ~70 % of the triangles and axis-aligned boxes for the rest, two emissive panels, sun and sky."""
    rng = PCG32(seed, stream=11)
    mats = [Material("ground", (0.55, 0.52, 0.48, 1.0)), Material("stone", (0.78, 0.76, 0.7, 1.0)),
            Material("lamp0", (0.9, 0.9, 0.9, 1.0), emissive=(10.0, 9.5, 8.5)),
            Material("lamp1", (0.9, 0.9, 0.9, 1.0), emissive=(8.0, 9.0, 10.0))]
    nbox_mats = 6
    for k in range(nbox_mats):
        mats.append(Material(f"box{k}", (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), 1.0)))
    b = Builder(mats)
    h = area / 2
    cells = 8
    step = area / cells
    b.mat = 0
    for j in range(cells):
        for i in range(cells):
            x0, z0 = -h + i * step, -h + j * step
            b.quad([x0, 0, z0 + step], [x0 + step, 0, z0 + step], [x0 + step, 0, z0], [x0, 0, z0])
    col_budget = int(0.7 * target_tris)
    seg, rings = 16, 8
    per_col = 2 * seg * rings
    ncol = max(1, col_budget // per_col)
    b.mat = 1
    for _ in range(ncol):
        cx, cz = rng.uniform(-h + 1, h - 1), rng.uniform(-h + 1, h - 1)
        if abs(cx) < 2 and abs(cz) < 2:
            cx += 4.0
        pos, nrm, tris = _cylinder(cx, cz, rng.uniform(0.15, 0.5), rng.uniform(2.0, 8.0), seg, rings)
        b.mesh(pos, nrm, tris)
    nbox = max(1, (target_tris - 2 * cells * cells - ncol * per_col) // 12)
    for _ in range(nbox):
        b.mat = 4 + int(rng.uniform(0, nbox_mats - 1e-9))
        c = [rng.uniform(-h + 1, h - 1), rng.uniform(0.1, 5.0), rng.uniform(-h + 1, h - 1)]
        if abs(c[0]) < 1.5 and abs(c[2]) < 1.5:
            c[0] += 3.0
        b.box(c, [rng.uniform(0.1, 1.0), rng.uniform(0.1, 1.0), rng.uniform(0.1, 1.0)])
    for k in range(2):
        b.mat = 2 + k
        cx, cz = rng.uniform(-h / 2, h / 2), rng.uniform(-h / 2, h / 2)
        b.quad_facing([cx - 1, 6.0, cz + 1], [cx + 1, 6.0, cz + 1], [cx + 1, 6.0, cz - 1], [cx - 1, 6.0, cz - 1], (0, -1, 0))
    cam = Camera((0.0, 1.7, 0.0), (10.0, 1.2, 3.0), 60, 0.05)
    from .frame import SUN_E, SKY
    return b.scene(name or f"mix-{seed}", cam, sun_dir=(-0.3, 1.0, 0.4), sun_e=SUN_E, sky=SKY)


def batch_spec(seed: int) -> dict:
    """One solve of the uneven batch: triangle count log-uniform 5k-500k, a clipmap of 32^3-256^3 voxels per level
    with 1-4 levels, a resolution of 320x180-1920x1080 (16:9) and 2-5 cascades, all drawn from PCG32(seed)."""
    rng = PCG32(seed, stream=23)
    tris = int(math.exp(rng.uniform(math.log(5_000), math.log(500_000))))
    G = [4, 8, 16, 32][int(rng.uniform(0, 4 - 1e-9))]
    levels = 1 + int(rng.uniform(0, 4 - 1e-9))
    W = 320 + 16 * int(rng.uniform(0, (1920 - 320) / 16 + 1 - 1e-9))
    H = max(180, (W * 9 // 16) // 4 * 4)
    cascades = 2 + int(rng.uniform(0, 4 - 1e-9))
    v0 = [0.1, 0.15, 0.2][int(rng.uniform(0, 3 - 1e-9))]
    return {"seed": seed, "tris": tris, "G": G, "levels": levels, "width": W, "height": H, "cascades": cascades, "v0": v0}


def textured_scene(size: int = 64) -> Scene:
    """The room of 60 boxes with base colour textures: every box face mapped to a coloured stripe image (layer 1),
    and four alpha-masked panels in the room (a cut-out lattice, layer 2: alpha 0 in the holes, cutoff 0.5), so the
    voxel passes' alpha test, the albedo sampling and the rasters' alpha test all see texels.  uvs: each quad's corners
    (0,0) (2,0) (2,2) (0,2) — repeat addressing tiles the image twice."""
    import dataclasses
    s = room_scene(0, n_boxes=60)
    nv = s.positions.shape[0]
    corners = np.array([[0.0, 0.0], [2.0, 0.0], [2.0, 2.0], [0.0, 2.0]], np.float32)
    uvs = np.tile(corners, (nv // 4 + 1, 1))[:nv]
    # layer 1: stripes of four colours; layer 2: a lattice, opaque bars of size/8 texels every size/2, alpha 0 between
    # (holes wider than a level-3 texel, so the voxel passes' sampling at level 3 + L still sees them)
    img = np.zeros((2, size, size, 4), np.uint8)
    x = np.arange(size)
    pal = np.array([[230, 60, 40], [40, 200, 80], [50, 90, 230], [240, 220, 60]], np.uint8)
    img[0, :, :, :3] = pal[(x[None, :] * 4 // size) % 4]
    img[0, :, :, 3] = 255
    bars = ((x[:, None] % (size // 2)) < size // 8) | ((x[None, :] % (size // 2)) < size // 8)
    img[1, :, :, :3] = 200
    img[1, :, :, 3] = np.where(bars, 255, 0)
    mats = [dataclasses.replace(m, base_color_tex=1) if m.name.startswith("box") else m for m in s.materials]
    # the panels: 1.5 m squares standing in the room
    b = Builder([Material("panel", (0.9, 0.9, 0.9, 1.0), flags=FLAG_ALPHA_MASK, alpha_cutoff=0.5,
                          base_color_tex=2)])
    for k, (cx, cz) in enumerate(((1.0, 1.0), (-2.0, 0.5), (0.5, -2.5), (2.5, -1.0))):
        b.quad([cx - 0.75, 0.2, cz], [cx + 0.75, 0.2, cz], [cx + 0.75, 1.7, cz], [cx - 0.75, 1.7, cz])
    panel = b.scene("panels", s.camera)
    pos = np.concatenate([s.positions, panel.positions]).astype(np.float32)
    nrm = np.concatenate([s.normals, panel.normals]).astype(np.float32)
    ptri = panel.tri.astype(np.int64).copy()
    ptri[:, :3] += nv
    ptri[:, 3] = len(mats)
    tri = np.concatenate([s.tri.astype(np.int64), ptri]).astype(np.uint32)
    puv = np.tile(corners, (panel.positions.shape[0] // 4, 1))
    return dataclasses.replace(s, name="room-textured", positions=pos, normals=nrm, tri=tri,
                               materials=mats + list(panel.materials), uvs=np.concatenate([uvs, puv]).astype(np.float32),
                               textures=img)
