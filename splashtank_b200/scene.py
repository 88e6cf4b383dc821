"""Scene and keyframe layer above the per-step call (src/shared.js:503-637), host side.

SceneRunner turns object states into the collider records of one step, with each collider's velocity and angular
velocity taken from its pose change since the previous step, then calls sim.step(dt, {...par, cols}) exactly as
SceneRunner.step does (src/shared.js:527-550). keyPose interpolates keyframes (src/shared.js:608-621).

Collider shapes are signed distance grids, the one collider form the reference's FLIP solver reads (packColliders,
src/gpu.js:42-70). sphere_sdf and box_sdf sample the exact distance of a sphere or a box on such a grid.
"""
import math

import numpy as np


def euler_mat(rx, ry, rz):
    """R = Rz * Ry * Rx, row major (eulerMat, src/shared.js:9-14)."""
    cx, sx, cy, sy, cz, sz = math.cos(rx), math.sin(rx), math.cos(ry), math.sin(ry), math.cos(rz), math.sin(rz)
    return [cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx,
            sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx,
            -sy, cy * sx, cy * cx]


def key_pose(keys, t, smooth=True):
    """Pose at time t from keyframes sorted by t (keyPose, src/shared.js:608-621): Catmull-Rom or linear."""
    n = len(keys)
    if t <= keys[0]["t"]:
        return dict(keys[0])
    if t >= keys[n - 1]["t"]:
        return dict(keys[n - 1])
    i = 0
    while i < n - 2 and t >= keys[i + 1]["t"]:
        i += 1
    a, b = keys[i], keys[i + 1]
    u = (t - a["t"]) / max(b["t"] - a["t"], 1e-6)
    p0 = keys[i - 1] if i > 0 else a
    p3 = keys[i + 2] if i + 2 < n else b
    u2, u3 = u * u, u * u * u

    def f(k):
        A, B, P0, P3 = a.get(k, 0), b.get(k, 0), p0.get(k, 0), p3.get(k, 0)
        if not smooth:
            return A + (B - A) * u
        return 0.5 * ((2 * A) + (-P0 + B) * u + (2 * P0 - 5 * A + 4 * B - P3) * u2 + (-P0 + 3 * A - 3 * B + P3) * u3)

    return dict(t=t, x=f("x"), y=f("y"), z=f("z"), rx=f("rx"), yaw=f("yaw"), rz=f("rz"))


def _grid(lo, hi, cell):
    n = [int(math.ceil((hi[a] - lo[a]) / cell)) + 1 for a in range(3)]
    ax = [lo[a] + cell * np.arange(n[a]) for a in range(3)]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return n, X, Y, Z


def sphere_sdf(r, cell, sid, margin=None):
    """Distance grid of a sphere of radius r centred on the collider position (x fastest)."""
    m = margin if margin is not None else 3 * cell
    lo = [-(r + m)] * 3
    n, X, Y, Z = _grid(lo, [r + m] * 3, cell)
    data = np.sqrt(X * X + Y * Y + Z * Z) - r
    return dict(id=sid, dims=n, origin=lo, cell=cell, data=data.astype(np.float32).ravel())


def box_sdf(hx, hy, hz, cell, sid, margin=None):
    """Distance grid of a box with half extents (hx, hy, hz) centred on the collider position."""
    m = margin if margin is not None else 3 * cell
    lo = [-(hx + m), -(hy + m), -(hz + m)]
    n, X, Y, Z = _grid(lo, [hx + m, hy + m, hz + m], cell)
    qx, qy, qz = np.abs(X) - hx, np.abs(Y) - hy, np.abs(Z) - hz
    out = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2 + np.maximum(qz, 0) ** 2)
    inside = np.minimum(np.maximum(qx, np.maximum(qy, qz)), 0.0)
    return dict(id=sid, dims=n, origin=lo, cell=cell, data=(out + inside).astype(np.float32).ravel())


class SceneRunner:
    """SceneRunner.step (src/shared.js:525-550) for mesh colliders: states are dicts with id, sdf, x, y, z, rx, yaw, rz."""

    def __init__(self, sim):
        self.sim = sim
        self.prev = {}

    def colliders(self, dt, states, col_max=20.0):
        lim2 = col_max ** 2
        cols = []
        for o in states:
            R = euler_mat(o.get("rx", 0), o.get("yaw", 0), o.get("rz", 0))
            p = self.prev.get(o["id"])
            self.prev[o["id"]] = dict(x=o["x"], y=o["y"], z=o["z"], R=R)
            c = dict(sdf=o["sdf"], x=o["x"], y=o["y"], z=o["z"], R=R, vx=0.0, vy=0.0, vz=0.0, wx=0.0, wy=0.0, wz=0.0)
            if p:
                vx, vy, vz = (o["x"] - p["x"]) / dt, (o["y"] - p["y"]) / dt, (o["z"] - p["z"]) / dt
                if vx * vx + vy * vy + vz * vz < lim2:
                    c.update(vx=vx, vy=vy, vz=vz)
                P = p["R"]
                d = [0.0] * 9   # dR = R * Rprev^T
                for r in range(3):
                    for q in range(3):
                        d[r * 3 + q] = R[r * 3] * P[q * 3] + R[r * 3 + 1] * P[q * 3 + 1] + R[r * 3 + 2] * P[q * 3 + 2]
                wx, wy, wz = (d[7] - d[5]) / (2 * dt), (d[2] - d[6]) / (2 * dt), (d[3] - d[1]) / (2 * dt)
                if wx * wx + wy * wy + wz * wz < lim2:
                    c.update(wx=wx, wy=wy, wz=wz)
            cols.append(c)
        return cols

    def step(self, dt, states, par):
        par = dict(par)
        par["cols"] = self.colliders(dt, states, par.get("colMax", 20.0))
        return self.sim.step(dt, par)
