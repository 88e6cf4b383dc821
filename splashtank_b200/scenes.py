"""Seeded synthetic scenes for the benchmark and parity workloads.

The reference seeds water with lattice points and an unseeded +-4% jitter (FluidSim.fillBox, src/shared.js:285-291).
The workloads here need reproducible inputs, so particles are placed 8 per cell (2 x 2 x 2 sub-cells of spacing d,
ratio 2), each uniformly jittered inside its sub-cell from a seeded numpy generator.

Coordinates: a workload stated on [0, W] x [0, H] x [0, D] maps to the reference box [-W/2, W/2] x [0, H] x [-D/2, D/2]
(src/flip/sim.js:53) by x_ref = x - W/2, z_ref = z - D/2.
"""
import math

import numpy as np


def seed_cells(cells_ijk, h, rng, x0, y0, z0, chunk=1 << 20):
    """8 jittered particles per cell: one per 2 x 2 x 2 sub-cell. cells_ijk is (n, 3) int; returns (8n, 3) float32.
    Cells are processed in chunks so a 256^3 tank (about 40M particles) needs little temporary memory."""
    d = h / 2.0
    sub = np.array([[sx, sy, sz] for sz in (0, 1) for sy in (0, 1) for sx in (0, 1)], np.float64)   # x fastest
    out = np.empty((len(cells_ijk) * 8, 3), np.float32)
    for a in range(0, len(cells_ijk), chunk):
        c = cells_ijk[a:a + chunk]
        base = c.astype(np.float64)[:, None, :] * h + sub[None, :, :] * d
        p = (base + rng.random(base.shape) * d).reshape(-1, 3)
        p[:, 0] += x0
        p[:, 1] += y0
        p[:, 2] += z0
        out[a * 8:(a + len(c)) * 8] = p
    return out


def box_cells(n_xyz, pred):
    """Cells (i, j, k) of an n_xyz grid whose centre (in cell units) satisfies pred(ci, cj, ck); k outer, i inner."""
    nx, ny, nz = n_xyz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m = pred(i + 0.5, j + 0.5, k + 0.5)
    return np.stack([i[m], j[m], k[m]], 1)


def ocean_tank(n=32, seed=5, level=0.3, layer=0.12, height=0.05, length=0.35, band=3.0, spray_cap=20000):
    """An ocean scene: waves (24 linear waves, significant height `height`, peak wavelength `length`) at mean level
    `level`, held to the side walls by a boundary layer `layer` wide; narrow band of `band` cells. The particles start
    in the band under the mean level (8 per cell, seeded jitter, at rest) inside the boundary's inner half; the depth
    field and the starting velocity come from the ocean itself (fillPhi and phiInitAll on a restart). Whitewater with
    the app's settings, the air field and gusts."""
    h = 1.0 / n
    rng = np.random.default_rng(seed)
    lw = lambda ci, ck: 1.0 - np.minimum(np.minimum(ci * h, 1.0 - ci * h), np.minimum(ck * h, 1.0 - ck * h)) / layer   # noqa: E731
    cells = box_cells((n, n, n), lambda ci, cj, ck: (cj * h < level) & (cj * h > level - band * h) & (lw(ci, ck) < 0.5))
    pos = seed_cells(cells, h, rng, -0.5, 0.0, -0.5)
    ocean = dict(on=True, level=level, layer=layer, length=length, height=height, dir=30.0, spread=20.0, seed=3)
    opts = dict(g=9.81, flip=0.95, comp=6.0, iters=30, vmax=50.0, drag=0.3, gust=1.0, tear=2.0, spr=dict(APP_SPRAY, min=0.25),
                nb=dict(on=True, band=band), ocean=ocean, air=dict(on=True, couple=3.0, decay=0.6))
    return dict(d=h / 2.0, ratio=2.0, size=(1.0, 1.0, 1.0), open=0, pos=pos, vel=np.zeros_like(pos), dt=1.0 / 240.0, opts=opts,
                spray_cap=spray_cap, spare=len(pos) // 2 + 4000, name="ocean_tank_%d" % n)


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


# the app's whitewater and solver settings (simPar, src/app/01-draw.js:55-63, defaults src/app/00-state.js:8-15)
APP_SPRAY = dict(rate=24.0, min=2.5, life=1.2, mist=0.3, drag=1.0, mdrag=5.0, ww=dict(foamLife=3.0, rise=0.4, crest=1.0, impact=0.25))


class WaveTank:
    """Full-feature wave tank on an n^3 grid over the unit box (256^3 is the benchmark workload).

    Water fills the lower 30% (cell centres below y = 0.3) in front of a piston; 8 particles per cell, seeded jitter.
    Piston: a box collider whose front face moves as xf(t) = -0.44 + 0.05 sin(2 pi 0.5 t) (0.5 Hz, amplitude 0.05);
    the block reaches past the -x wall, so no water is trapped behind it. Sphere: r = 0.1 on a linear keyframed path from
    y = 0.55 down through the surface to y = 0.12 over the 200 steps. Narrow band on at full depth (band 1e4: particles
    all the way down, depth field and kept grid velocity maintained, refill of thin calm cells); whitewater with the app's
    settings except an emission speed threshold of 0.25 m/s so the slow piston waves throw off points; the air field on
    with the app's coupling 3 and decay 0.6 (src/app/00-state.js:9, so spray and mist drift with the air the water and
    spray drag along); drips on with the app's rate 2 and drying time 3 s (the colliders drip after they leave the
    water); air drag 0.3 with gusts, sheet tearing below 2 particles, 30 SOR iterations, dt = 1/240.
    """

    def __init__(self, n=256, seed=7, spray_cap=4_000_000, band=1e4, steps=200):
        self.n = n
        self.h = 1.0 / n
        self.d = self.h / 2.0
        self.dt = 1.0 / 240.0
        self.steps = steps
        self.spray_cap = spray_cap
        self.band = band
        self.xf0 = -0.44
        rng = np.random.default_rng(seed)
        h = self.h
        cells = box_cells((n, n, n), lambda ci, cj, ck: (cj * h < 0.3) & (ci * h - 0.5 > self.xf0 + 0.5 * h))
        self.pos = seed_cells(cells, h, rng, -0.5, 0.0, -0.5)
        self.vel = np.zeros_like(self.pos)
        from .scene import box_sdf, sphere_sdf
        self.piston_sdf = box_sdf(0.1, 0.35, 0.53, 0.01, sid=1)
        self.sphere_sdf = sphere_sdf(0.1, 0.01, sid=2)
        T = steps * self.dt
        self.sphere_keys = [dict(t=0.0, x=0.15, y=0.55, z=0.0), dict(t=T, x=0.15, y=0.12, z=0.0)]
        self.opts = dict(g=9.81, flip=0.95, comp=6.0, iters=30, vmax=50.0, drag=0.3, gust=1.0, foamSens=1.0, foamTau=1.2,
                         tear=2.0, vs=1.0, colMax=100.0, spr=dict(APP_SPRAY, min=0.25), nb=dict(on=True, band=band),
                         air=dict(on=True, couple=3.0, decay=0.6), drip=dict(on=True, rate=2.0, dry=3.0))
        self.fill_box = (self.xf0, -1e4, -1e4, 1e4, 0.3, 1e4)   # x0, y0, z0, x1, y1, z1 (faces on walls pushed out)

    def states(self, t):
        from .scene import key_pose
        xf = self.xf0 + 0.05 * math.sin(2 * math.pi * 0.5 * t)
        s = key_pose(self.sphere_keys, t, smooth=False)
        return [dict(id=1, sdf=self.piston_sdf, x=xf - 0.1, y=0.3, z=0.0),
                dict(id=2, sdf=self.sphere_sdf, x=s["x"], y=s["y"], z=s["z"])]

    def spare(self):
        """Parked slots the narrow band refills from (nbSeed keeps ceil(0.35 * seeded) + 4000, src/shared.js:846-848, sized
        for a thin band). At full depth almost no cell runs short, so this tank keeps 2% + 4000."""
        return int(math.ceil(0.02 * len(self.pos))) + 4000

    def make(self, cls, **kw):
        """A simulator (FlipSim or a class with the same constructor) loaded with this tank."""
        spare = self.spare()
        sim = cls(self.d, len(self.pos) + spare, size=(1.0, 1.0, 1.0), ratio=2.0, spray_cap=self.spray_cap, **kw)
        sim.add_many(self.pos, self.vel)
        park = np.zeros((spare, 3), np.float32)
        park[:, 1] = -1.0e6
        sim.add_many(park)
        sim.nb_fills(boxes=[self.fill_box], mode=1)
        return sim


def splash_blobs(n=512, seed=11, blobs=None, sigma=(0.025, 0.07), level=0.5):
    """Pressure-solve workload: fluid where a sum of seeded Gaussian blobs exceeds level (splash-shaped, merged), inside
    solid walls; rhs is the divergence of a seeded random face-velocity field on the fluid cells. Returns (type, rhs) as
    (n, n, n) arrays indexed [k][j][i]: uint8 0 air / 1 fluid, float64. About 20% of the 8^3 tiles hold fluid."""
    rng = np.random.default_rng(seed)
    k_blobs = blobs if blobs is not None else 120
    c = rng.uniform(0.12, 0.88, (k_blobs, 3))
    s = rng.uniform(sigma[0], sigma[1], k_blobs)
    f = np.zeros((n, n, n), np.float32)
    h = 1.0 / n
    for (cx, cy, cz), sg in zip(c, s):
        r = 2.6 * sg
        lo = [max(0, int((q - r) / h)) for q in (cx, cy, cz)]
        hi = [min(n, int((q + r) / h) + 1) for q in (cx, cy, cz)]
        xs = ((np.arange(lo[0], hi[0]) + 0.5) * h - cx).astype(np.float32)
        ys = ((np.arange(lo[1], hi[1]) + 0.5) * h - cy).astype(np.float32)
        zs = ((np.arange(lo[2], hi[2]) + 0.5) * h - cz).astype(np.float32)
        inv = np.float32(-0.5 / (sg * sg))
        g = np.exp(zs[:, None, None] ** 2 * inv) * np.exp(ys[None, :, None] ** 2 * inv) * np.exp(xs[None, None, :] ** 2 * inv)
        f[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += g
    cell_type = (f > level).astype(np.uint8)
    del f
    rhs = np.zeros((n, n, n), np.float64)
    slab = 32
    for z0 in range(0, n, slab):
        z1 = min(n, z0 + slab)
        r2 = np.random.default_rng([seed, z0])
        u = r2.uniform(-1, 1, (z1 - z0, n, n + 1))
        v = r2.uniform(-1, 1, (z1 - z0, n + 1, n))
        w = r2.uniform(-1, 1, (z1 - z0 + 1, n, n))
        rhs[z0:z1] = (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:] - w[:-1])
    rhs[cell_type != 1] = 0.0
    return cell_type, rhs


TANK_EDGES = (32, 48, 64, 96, 128)


class BatchTanks:
    """Many independent tanks of uneven size: each axis edge (cells) drawn uniformly from TANK_EDGES, cell size 1/64, a
    random axis-aligned fluid box filling 20-60% of the tank (8 particles per cell, seeded jitter) that falls from where
    it is placed, and one static SDF sphere (radius 8-20% of the shortest extent) at a random place. Solid walls, FLIP
    0.95, gravity 9.81, 30 SOR iterations, dt = 1/240; no whitewater or narrow band."""

    def __init__(self, count=64, seed=5, h=1.0 / 64.0, steps=100, edges=TANK_EDGES):
        self.h = h
        self.dt = 1.0 / 240.0
        self.steps = steps
        rng = np.random.default_rng(seed)
        self.tanks = []
        for k in range(count):
            e = [int(x) for x in rng.choice(edges, 3)]
            f = float(rng.uniform(0.2, 0.6))
            ax = float(rng.uniform(f, 1.0))
            ay = float(rng.uniform(f / ax, 1.0))
            az = f / (ax * ay)
            frac = (ax, ay, az)
            lo = [float(rng.uniform(0.0, 1.0 - a)) for a in frac]
            size = [x * h for x in e]
            r = float(rng.uniform(0.08, 0.2)) * min(size)
            c = [float(rng.uniform(r, sz - r)) - (sz / 2.0 if a != 1 else 0.0) for a, sz in enumerate(size)]
            self.tanks.append(dict(edges=e, size=size, fill=frac, lo=lo, sphere=(c[0], c[1], c[2], r), seed=int(rng.integers(1 << 31))))
        self.opts = dict(g=9.81, flip=0.95, comp=6.0, iters=30, vmax=14.0)

    def particles(self, k):
        t = self.tanks[k]
        e, h = t["edges"], self.h
        lo = [t["lo"][a] * e[a] for a in range(3)]
        hi = [lo[a] + t["fill"][a] * e[a] for a in range(3)]
        cells = box_cells(e, lambda ci, cj, ck: (ci >= lo[0]) & (ci < hi[0]) & (cj >= lo[1]) & (cj < hi[1]) & (ck >= lo[2]) & (ck < hi[2]))
        rng = np.random.default_rng(t["seed"])
        size = t["size"]
        return seed_cells(cells, h, rng, -size[0] / 2.0, 0.0, -size[2] / 2.0)

    def cost(self, k, n_particles=None):
        """Work estimate of a tank (cells + particles), for splitting tanks over GPUs."""
        t = self.tanks[k]
        cells = t["edges"][0] * t["edges"][1] * t["edges"][2]
        n = n_particles if n_particles is not None else 8 * cells * t["fill"][0] * t["fill"][1] * t["fill"][2]
        return float(cells + n)

    def make(self, k, cls, **kw):
        from .scene import sphere_sdf
        t = self.tanks[k]
        pos = self.particles(k)
        sim = cls(self.h / 2.0, max(len(pos), 1), size=tuple(t["size"]), ratio=2.0, **kw)
        sim.add_many(pos, np.zeros_like(pos))
        sim.sphere = sphere_sdf(t["sphere"][3], self.h, sid=100 + k)
        return sim, len(pos)

    def step_opts(self, k, sim, runner):
        """Tank k's options for one step: its static sphere as the one collider (SceneRunner records)."""
        t = self.tanks[k]
        st = [dict(id=100 + k, sdf=sim.sphere, x=t["sphere"][0], y=t["sphere"][1], z=t["sphere"][2])]
        o = dict(self.opts)
        o["cols"] = runner.colliders(self.dt, st, 20.0)
        return o


def splat_density(pos, n):
    """Cell-centred trilinear density of particles on an n^3 grid over the unit box (x fastest), corners clamped."""
    g = pos.astype(np.float64) * n - 0.5
    f0 = np.floor(g)
    fr = g - f0
    i0 = f0.astype(np.int64)
    rho = np.zeros(n ** 3, np.float64)
    for c in range(8):
        o = np.array([(c >> d) & 1 for d in range(3)])
        ii = np.clip(i0 + o, 0, n - 1)
        w = np.prod(np.where(o == 1, fr, 1.0 - fr), axis=1)
        rho += np.bincount(ii[:, 0] + n * (ii[:, 1] + n * ii[:, 2]), weights=w, minlength=n ** 3)
    return rho.astype(np.float32)


class DiffDam:
    """Differentiation workload: n^3 dam break on the unit box (water where x < 0.4, y < 0.6, 8 particles per cell,
    seeded jitter) with a moving box collider (half extents 0.06 x 0.12 x 0.25) whose centre follows 8 keyframes from
    (0.75, 0.3, 0.5) towards the water; loss against a seeded target density: the starting water moved by a seeded
    offset. Parameters: the keyframes (24) then the initial fluid velocity (3)."""

    def __init__(self, n=128, seed=21, steps=32, ckpt=8, fx=0.4, fy=0.6, jitter=True):
        """jitter=False puts every particle at the centre of its sub-cell, a quarter cell from every face where the
        trilinear weights bend (for finite differences that cross none of them)."""
        self.n, self.steps, self.ckpt = n, steps, ckpt
        h = 1.0 / n
        rng = np.random.default_rng(seed)
        cells = box_cells((n, n, n), lambda ci, cj, ck: (ci * h < fx) & (cj * h < fy))
        if jitter:
            self.pos = seed_cells(cells, h, rng, 0.0, 0.0, 0.0)
        else:
            sub = np.array([[sx, sy, sz] for sz in (0, 1) for sy in (0, 1) for sx in (0, 1)], np.float64)
            self.pos = ((cells.astype(np.float64)[:, None, :] + (sub[None] + 0.5) * 0.5) * h).reshape(-1, 3).astype(np.float32)
        keys = np.array([[0.75 - 0.04 * k, 0.3, 0.5] for k in range(8)], np.float64)
        self.params = np.concatenate([keys.ravel(), [0.2, 0.0, 0.0]])
        off = np.array([rng.uniform(0.02, 0.08), -rng.uniform(0.0, 0.05), rng.uniform(-0.03, 0.03)])
        moved = np.clip(self.pos + off.astype(np.float32), 0.5 * h, 1 - 0.5 * h)
        self.target = splat_density(moved, n)

    def make(self, **kw):
        from .diff import DiffRollout
        return DiffRollout(self.n, self.pos, self.target, self.steps, ckpt_every=self.ckpt, **kw)
