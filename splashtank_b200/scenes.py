"""Seeded synthetic scenes for the benchmark and parity workloads.

The reference seeds water with lattice points and an unseeded +-4% jitter (FluidSim.fillBox, src/shared.js:285-291).
The workloads here need reproducible inputs, so particles are placed 8 per cell (2 x 2 x 2 sub-cells of spacing d,
ratio 2), each uniformly jittered inside its sub-cell from a seeded numpy generator.

Coordinates: a workload stated on [0, W] x [0, H] x [0, D] maps to the reference box [-W/2, W/2] x [0, H] x [-D/2, D/2]
(src/flip/sim.js:53) by x_ref = x - W/2, z_ref = z - D/2.
"""
import numpy as np


def seed_cells(cells_ijk, h, rng, x0, y0, z0):
    """8 jittered particles per cell: one per 2 x 2 x 2 sub-cell. cells_ijk is (n, 3) int; returns (8n, 3) float32."""
    d = h / 2.0
    sub = np.array([[sx, sy, sz] for sz in (0, 1) for sy in (0, 1) for sx in (0, 1)], np.float64)   # x fastest
    base = cells_ijk.astype(np.float64)[:, None, :] * h + sub[None, :, :] * d
    u = rng.random(base.shape)
    p = base + u * d
    p = p.reshape(-1, 3)
    p[:, 0] += x0
    p[:, 1] += y0
    p[:, 2] += z0
    return p.astype(np.float32)


def box_cells(n_xyz, pred):
    """Cells (i, j, k) of an n_xyz grid whose centre (in cell units) satisfies pred(ci, cj, ck); k outer, i inner."""
    nx, ny, nz = n_xyz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m = pred(i + 0.5, j + 0.5, k + 0.5)
    return np.stack([i[m], j[m], k[m]], 1)


def dam_break(n=64, seed=1234, fx=0.4, fy=0.6):
    """Plain FLIP dam break: n^3 MAC grid (dx = 1/n) in 8^3 blocks, solid walls; fluid where the cell centre has
    x < fx and y < fy (all z); 8 particles per cell, seeded jitter. FLIP 0.97, gravity 9.81, dt 1/240, 50 red-black SOR
    iterations at omega 1.7; no whitewater, narrow band or colliders."""
    h = 1.0 / n
    rng = np.random.default_rng(seed)
    cells = box_cells((n, n, n), lambda ci, cj, ck: (ci * h < fx) & (cj * h < fy))
    pos = seed_cells(cells, h, rng, -0.5, 0.0, -0.5)
    return dict(d=h / 2.0, ratio=2.0, size=(1.0, 1.0, 1.0), open=0, pos=pos, vel=np.zeros_like(pos), dt=1.0 / 240.0,
                opts=dict(g=9.81, flip=0.97, iters=50, omega=1.7, comp=6.0, vmax=14.0), steps=100, name="dam_break_%d" % n)
