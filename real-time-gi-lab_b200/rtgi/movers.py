"""Moving rigid boxes added to a static scene (no counterpart in the reference, whose moving objects go through its
dynamic layer, dynlayer.ts; here they are re-posed on the host and the clipmap is rebuilt from all triangles every
frame, the reference's full-dynamic rebuild, voxel.ts:14-15).

The boxes are appended after the scene's own triangles as one extra material, so their vertices are one contiguous
range: a frame re-poses them with one gi_scene_update_vertices call."""
from __future__ import annotations

import math

import numpy as np

from . import scenes


class MovingObjects:
    """Rigid boxes at the end of a scene's vertex array: rest vertices, and a pose (rotation about y through the
    box centre, then a translation along a constant velocity, wrapped into a rectangle of the ground plane) at time t."""

    def __init__(self, first_vertex: int, pos: np.ndarray, nrm: np.ndarray, centres: np.ndarray, vel: np.ndarray,
                 omega: np.ndarray, area=(0.0, 0.0, 20.0, 20.0)):
        self.first = first_vertex
        self.rest_pos = pos.astype(np.float64)
        self.rest_nrm = nrm.astype(np.float64)
        self.centres = centres
        self.vel = vel
        self.omega = omega
        self.area = area            # (centre x, centre z, half extent x, half extent z)
        self.per = pos.shape[0] // max(1, centres.shape[0])

    def transforms(self, t: float) -> np.ndarray:
        """(n, 12) float32 row-major [R | c(t) - R c0] per object: the pose at t as a transform of the rest vertices
        (what pose() computes, for gi_scene_rigid_upload)."""
        k = self.centres.shape[0]
        ax, az, hx, hz = self.area
        c = self.centres + self.vel * t
        c[:, 0] = (c[:, 0] - ax + hx) % (2 * hx) - hx + ax
        c[:, 2] = (c[:, 2] - az + hz) % (2 * hz) - hz + az
        a = self.omega * t
        ca, sa = np.cos(a), np.sin(a)
        m = np.zeros((k, 12), np.float64)
        m[:, 0], m[:, 2], m[:, 5], m[:, 8], m[:, 10] = ca, sa, 1.0, -sa, ca
        c0 = self.centres
        m[:, 3] = c[:, 0] - (ca * c0[:, 0] + sa * c0[:, 2])
        m[:, 7] = c[:, 1] - c0[:, 1]
        m[:, 11] = c[:, 2] - (-sa * c0[:, 0] + ca * c0[:, 2])
        return m.astype(np.float32)

    def pose(self, t: float):
        k = self.centres.shape[0]
        ax, az, hx, hz = self.area
        c = self.centres + self.vel * t
        c[:, 0] = (c[:, 0] - ax + hx) % (2 * hx) - hx + ax
        c[:, 2] = (c[:, 2] - az + hz) % (2 * hz) - hz + az
        a = self.omega * t
        ca, sa = np.cos(a), np.sin(a)
        rel = self.rest_pos.reshape(k, self.per, 3) - self.centres[:, None, :]
        x, y, z = rel[..., 0], rel[..., 1], rel[..., 2]
        pos = np.stack([c[:, None, 0] + ca[:, None] * x + sa[:, None] * z, c[:, None, 1] + y,
                        c[:, None, 2] - sa[:, None] * x + ca[:, None] * z], -1).reshape(-1, 3)
        n = self.rest_nrm.reshape(k, self.per, 3)
        nrm = np.stack([ca[:, None] * n[..., 0] + sa[:, None] * n[..., 2], n[..., 1],
                        -sa[:, None] * n[..., 0] + ca[:, None] * n[..., 2]], -1).reshape(-1, 3)
        return pos.astype(np.float32), nrm.astype(np.float32)


def with_moving_boxes(base: scenes.Scene, n: int, rng: scenes.PCG32, area=(0.0, 0.0, 15.0, 15.0),
                      height=(0.2, 1.5), half_side=(0.1, 0.5), speed=(0.0, 2.0), colour=(0.8, 0.3, 0.2, 1.0)):
    """`base` with n boxes appended: centres uniform in the area rectangle at heights U(height), half sides
    U(half_side), horizontal velocities of speed U(speed) m/s in a uniform direction, spin U(-1, 1) rad/s.
    Returns (scene, MovingObjects)."""
    b = scenes.Builder(list(base.materials) + [scenes.Material("object", colour)])
    # the base geometry again, one index list per material, in its own triangle order
    b.pos = base.positions.astype(np.float64).reshape(-1).tolist()
    b.nrm = base.normals.astype(np.float64).reshape(-1).tolist()
    for m in range(len(base.materials)):
        rows = base.tri[base.tri[:, 3] == m, :3]
        b.idx[m] = rows.reshape(-1).tolist()
    first = len(b.pos) // 3
    b.mat = len(base.materials)
    ax, az, hx, hz = area
    centres, vel, omega = [], [], []
    for _ in range(n):
        c = [rng.uniform(ax - hx, ax + hx), rng.uniform(*height), rng.uniform(az - hz, az + hz)]
        hs = [rng.uniform(*half_side) for _ in range(3)]
        b.box(c, hs)
        sp, ang = rng.uniform(*speed), rng.uniform(0, 2 * math.pi)
        centres.append(c)
        vel.append([sp * math.cos(ang), 0.0, sp * math.sin(ang)])
        omega.append(rng.uniform(-1, 1))
    s = b.scene(base.name + f"-obj{n}", base.camera, sun_dir=base.sun_dir, sun_e=base.sun_e, sky=base.sky)
    objs = MovingObjects(first, s.positions[first:], s.normals[first:], np.array(centres), np.array(vel),
                         np.array(omega), (ax, az, hx + 5.0, hz + 5.0))
    return s, objs
