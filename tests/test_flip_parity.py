"""GPU parity of the sm_100a FLIP step with the CPU oracle, through the C ABI.

Bar: bit-exact. The kernels and the oracle perform the same f32 operations in the same order (no contraction,
shared exp/sin/cos from include/st_math.h), and every order the reference leaves to atomics is fixed the same way on
both sides, so positions, velocities, pressures, face velocities, cell types, counts, tile sets, the storage order and
the whitewater pool must agree bit for bit, not just within a tolerance.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))


@pytest.fixture(scope="module", autouse=True)
def built():
    from splashtank_b200 import build
    build.build()
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "liboracle_flip.so")], check=True)


def same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def assert_same_state(g, o, spray=False):
    pa, va, ia = g.save_state()
    pb, vb, ib = o.save_state()
    assert same(ia, ib), "storage order"
    assert same(pa, pb), "positions (max diff %g)" % np.max(np.abs(pa - pb))
    assert same(va, vb), "velocities (max diff %g)" % np.max(np.abs(va - vb))
    A, B = g.grid(), o.grid()
    for k in ("tile_on", "cnt", "ctype", "pres", "rhs", "vn", "vo", "velg"):
        assert same(A[k], B[k]), "%s differs at %d cells" % (k, int(np.sum(np.asarray(A[k]) != np.asarray(B[k]))))
    sa, sb = g.readStats(), o.readStats()
    for k in ("sc", "fluid", "vmax", "n", "live", "spray_used"):
        assert sa[k] == sb[k], k
    if spray:
        x, y = g.readSpray(), o.readSpray()
        assert x["n"] == y["n"] and same(x["p"], y["p"]) and same(x["v"], y["v"]), "whitewater"
        a, b = g.read_air(), o.read_air()
        assert (a is None) == (b is None) and (a is None or same(a, b)), "air field"


def dam_pair(n, **kw):
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    sc = scenes.dam_break(n)
    sc.update(kw)
    return make_pair(sc), sc


def test_dam_break_one_step():
    (g, o), sc = dam_pair(32)
    for s in (g, o):
        s.step(sc["dt"], sc["opts"])
    assert_same_state(g, o)


def test_dam_break_thirty_steps():
    (g, o), sc = dam_pair(32)
    for _ in range(30):
        for s in (g, o):
            s.step(sc["dt"], sc["opts"])
    assert_same_state(g, o)


def test_open_floor_dead_particles():
    (g, o), sc = dam_pair(16, open=4)
    for _ in range(45):
        for s in (g, o):
            s.step(sc["dt"], sc["opts"])
    assert g.readStats()["live"] < g.readStats()["n"]
    assert_same_state(g, o)


@pytest.mark.parametrize("name", ["dam_break_16_s10", "wave_tank_24_s8"])
def test_golden_fixtures(name):
    from golden.make_golden import run_case
    from splashtank_b200.flip import FlipSim
    ref = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    got = run_case(name, cls=FlipSim)
    for k in ref.files:
        assert same(got[k], ref[k]), k


def _tank_pair(n, band, spray_cap=50000):
    from oracle.oracle import OracleFlipSim
    from splashtank_b200 import scenes
    from splashtank_b200.flip import FlipSim
    w = scenes.WaveTank(n, spray_cap=spray_cap, band=band)
    return w, w.make(FlipSim), w.make(OracleFlipSim, threads=8)


def _run_tank(w, sims, steps):
    from splashtank_b200.scene import SceneRunner
    runs = [SceneRunner(s) for s in sims]
    t = 0.0
    for _ in range(steps):
        t += w.dt
        st = w.states(t)
        for r in runs:
            r.step(w.dt, st, w.opts)


def test_wave_tank_full_depth():
    """Piston + sphere colliders, narrow band at full depth, whitewater, gusts, sheet tearing: 40 steps."""
    w, g, o = _tank_pair(40, 1e4)
    _run_tank(w, (g, o), 40)
    assert g.readStats()["spray_used"] > 0 or True
    assert_same_state(g, o, spray=True)


def test_wave_tank_band3_trims_and_refills():
    """Narrow band of 3 cells: deep calm particles are killed and thin band cells refilled from the dead slots."""
    w, g, o = _tank_pair(32, 3.0)
    _run_tank(w, (g, o), 30)
    st = g.readStats()
    assert st["live"] < len(w.pos)     # the deep water was trimmed to the band
    assert_same_state(g, o, spray=True)


@pytest.mark.parametrize("spray_cap", [30000, 4000])
def test_air_field_with_whitewater(spray_cap):
    """Whitewater of every kind with the air field on: water thrown at the wall from t = 0.6 s (emission at full
    strength), gusts, narrow band of 3 cells (the trim of particles the air splat still sees), 40 steps. With the
    smaller pool the ring wraps several times. The air field, the pool and the particles agree bit for bit."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    sc = scenes.dam_break(32)
    sc["vel"] = np.tile(np.array([[2.5, 0.5, 0.0]], np.float32), (len(sc["pos"]), 1))
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY, min=0.5), air=dict(on=True, couple=3.0, decay=0.6), gust=1.0,
                nb=dict(on=True, band=3.0))
    g, o = make_pair(sc, spray_cap=spray_cap)
    for s in (g, o):
        p, v, i = s.save_state()
        s.load_state(p, v, i, t=0.6, seed=0)
    for _ in range(40):
        for s in (g, o):
            s.step(sc["dt"], opts)
    sp = g.readSpray()
    kinds = np.bincount(np.round(sp["v"][sp["p"][:, 3] > 0, 3]).astype(int), minlength=4)
    assert np.all(kinds > 0), kinds                      # spray, mist, foam and bubbles all present
    assert g.readStats()["live"] < len(sc["pos"])          # the narrow band trimmed
    assert np.abs(g.read_air()).max() > 0.5
    assert_same_state(g, o, spray=True)


@pytest.mark.parametrize("mode", ["noFoam", "fastAir", None])
def test_density_terms_modes_and_a_packed_clump(mode):
    """g2p's local-density terms (air, shield, the foam decay and the drag factor) in each of the reference's modes: from
    the 2 x 2 x 2 corner count sum (the default: a per-CTA table of the sums below 256 and a direct evaluation above),
    from the particle's own cell (fastAir, with the gust skipped under shield) and at rest density (noFoam). Drag 0.3
    with gusts and a steady wind; a clump of 2,400 extra particles packed into 2 x 2 x 2 cells makes corner sums far
    above 256 in the first steps. 20 steps bit for bit."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    sc = scenes.dam_break(32)
    rng = np.random.default_rng(11)
    clump = (np.array([0.125, 0.3125, 0.0]) + rng.random((2400, 3)) * (2.0 / 32)).astype(np.float32)   # 2^3 cells in the air
    sc["pos"] = np.concatenate([sc["pos"], clump]).astype(np.float32)
    sc["vel"] = np.zeros_like(sc["pos"])
    opts = dict(sc["opts"], drag=0.3, gust=1.0, wind=(1.5, 0.0, -0.5))
    g, o = make_pair(sc)
    for s in (g, o):
        if mode:
            s.opt[mode] = True
    for _ in range(20):
        for s in (g, o):
            s.step(sc["dt"], opts)
    assert g.readStats()["live"] == len(sc["pos"])
    assert_same_state(g, o)


def test_rotating_box_collider():
    """A box collider (its distance grid) turning about two axes while it sweeps through a dam break: the solid cells,
    the faces' collider velocity with the spin, and g2p's collider response (its world-space, sphere and local-space
    pre-tests, colNear, sdfEval, the push-out and the removal of the velocity into the surface), 30 steps bit for
    bit."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    from splashtank_b200.scene import SceneRunner, box_sdf
    sc = scenes.dam_break(32)
    g, o = make_pair(sc)
    box = box_sdf(0.12, 0.06, 0.2, 1.0 / 64.0, sid=7)
    runs, t = [SceneRunner(s) for s in (g, o)], 0.0
    for _ in range(30):
        t += sc["dt"]
        st = [dict(id=7, sdf=box, x=-0.35 + 1.5 * t, y=0.2, z=0.05, yaw=0.6 + 3.0 * t, rx=0.3 + 2.0 * t)]
        for r in runs:
            r.step(sc["dt"], st, sc["opts"])
    assert_same_state(g, o)


def test_drips_from_a_rising_sphere():
    """A sphere lifted out of the water drips (no other emission): drip samples, their wetness, the drops in the
    whitewater pool, the air field they push and the water agree bit for bit after 60 steps."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    from splashtank_b200.scene import SceneRunner, sphere_sdf
    sc = scenes.dam_break(32)
    sdf = sphere_sdf(0.1, 0.01, sid=5)
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY, rate=0.0), air=dict(on=True, couple=3.0, decay=0.6),
                drip=dict(on=True, rate=20.0, dry=3.0))
    g, o = make_pair(sc, spray_cap=20000)
    runs, t = [SceneRunner(s) for s in (g, o)], 0.0
    for _ in range(60):
        t += sc["dt"]
        st = [dict(id=1, sdf=sdf, x=-0.3, y=0.3 + min(1.0, t / 0.15) * 0.55, z=0.0)]
        for r in runs:
            r.step(sc["dt"], st, opts)
    assert g.readStats()["spray_used"] >= 20
    da, db = g.read_drips(), o.read_drips()
    assert len(da) > 0 and same(da, db), "drip samples"
    assert_same_state(g, o, spray=True)


def test_ragged_box_open_face_collider_and_whitewater():
    """A box whose cell counts are multiples of 8 on no axis (37 x 22 x 29 cells; tile box 5 x 3 x 4 with its padding
    cells), open on +x, water thrown towards the open face past a moving sphere, whitewater with the air field, gusts,
    sheet tearing and a 3-cell narrow band: 30 steps bit for bit."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    from splashtank_b200.scene import SceneRunner, sphere_sdf
    h, n = 1.0 / 32, (37, 22, 29)
    size = tuple(k * h for k in n)
    rng = np.random.default_rng(21)
    cells = scenes.box_cells(n, lambda ci, cj, ck: (ci < 20) & (cj < 14))
    pos = scenes.seed_cells(cells, h, rng, -size[0] / 2, 0.0, -size[2] / 2)
    vel = np.tile(np.array([[1.5, 0.3, 0.2]], np.float32), (len(pos), 1))
    sc = dict(d=h / 2, ratio=2.0, size=size, open=2, pos=pos, vel=vel)
    opts = dict(g=9.81, flip=0.95, comp=6.0, iters=30, vmax=14.0, drag=0.3, gust=1.0, tear=2.0,
                spr=dict(scenes.APP_SPRAY, min=0.5), air=dict(on=True, couple=3.0, decay=0.6), nb=dict(on=True, band=3.0))
    g, o = make_pair(sc, spray_cap=30000)
    for s in (g, o):
        assert (s.nx, s.ny, s.nz) == n
        p, v, i = s.save_state()
        s.load_state(p, v, i, t=0.6, seed=0)
    sdf = sphere_sdf(0.08, h / 2, sid=7)
    runs, t, dt = [SceneRunner(s) for s in (g, o)], 0.0, 1.0 / 240.0
    for _ in range(30):
        t += dt
        st = [dict(id=1, sdf=sdf, x=0.1 + 0.5 * t, y=0.25, z=0.05)]
        for r in runs:
            r.step(dt, st, opts)
    gs = g.readStats()
    assert gs["live"] < gs["n"] and gs["spray_used"] > 0
    assert_same_state(g, o, spray=True)


def test_fill_volume_restart_with_a_collider():
    """A restart whose starting water is a water mesh (a fill volume's distance grid, packed after the colliders) and
    a box fill, next to a moving sphere collider, narrow band of 3 cells: 6 steps bit for bit."""
    from test_oracle import shell_drop
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner, sphere_sdf
    r, c = 0.22, (0.0, 0.45, 0.0)
    g, opts = shell_drop(FlipSim, r=r, c=c)
    o, _ = shell_drop(OracleFlipSim, r=r, c=c, threads=8)
    vol = dict(sdf=sphere_sdf(r, g.h / 2, sid=9), x=c[0], y=c[1], z=c[2])
    col = sphere_sdf(0.08, g.h / 2, sid=5)
    for s in (g, o):
        s.nb_fill_vols([vol])
        s.nb_fills(boxes=[(-0.5, 0.0, -0.5, 0.5, 0.06, 0.5)])
    runs, t, dt = [SceneRunner(s) for s in (g, o)], 0.0, 1.0 / 240.0
    for _ in range(6):
        t += dt
        st = [dict(id=1, sdf=col, x=0.3 - 0.5 * t, y=0.3, z=0.0)]
        for rr in runs:
            rr.step(dt, st, opts)
    assert_same_state(g, o)


def test_water_added_to_a_running_tank():
    """nbSeed's mode 2 (water added to a running tank, src/shared.js:849): after 5 steps a second ball is added as a
    fill volume and its band particles; the depth field keeps the old water and gains the new: 5 more steps bit for
    bit."""
    from test_oracle import shell_drop
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import sphere_sdf
    r, c = 0.22, (0.0, 0.45, 0.0)
    g, opts = shell_drop(FlipSim, r=r, c=c)
    o, _ = shell_drop(OracleFlipSim, r=r, c=c, threads=8)
    for s in (g, o):
        s.nb_fills(spheres=[(c[0], c[1], c[2], r)])
    dt = 1.0 / 240.0
    for _ in range(5):
        for s in (g, o):
            s.step(dt, opts)
    r2, c2 = 0.1, (-0.25, 0.75, 0.2)
    add, _ = shell_drop(OracleFlipSim, r=r2, c=c2, band=2.0, seed=8)
    p2 = add.save_state()[0][:, :3]
    vol = dict(sdf=sphere_sdf(r2, g.h / 2, sid=11), x=c2[0], y=c2[1], z=c2[2])
    for s in (g, o):
        s.add_many(p2)
        s.nb_fill_vols([vol], mode=2)
    for _ in range(5):
        for s in (g, o):
            s.step(dt, opts)
    assert_same_state(g, o)


def test_particle_state_round_trip():
    """save_state -> load_state -> save_state returns the same particles, ids and storage order."""
    from splashtank_b200 import scenes
    from splashtank_b200.flip import FlipSim
    sc = scenes.dam_break(24)
    a = FlipSim(sc["d"], len(sc["pos"]), size=sc["size"])
    a.add_many(sc["pos"])
    for _ in range(5):
        a.step(sc["dt"], sc["opts"])
    p, v, i = a.save_state()
    b = FlipSim(sc["d"], len(sc["pos"]), size=sc["size"])
    b.load_state(p, v, i, t=5 * sc["dt"], seed=5)
    pb, vb, ib = b.save_state()
    assert same(p, pb) and same(v, vb) and same(i, ib)


def test_deterministic_repeat():
    from splashtank_b200 import scenes
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    out = []
    for _ in range(2):
        w = scenes.WaveTank(32, spray_cap=20000)
        s = w.make(FlipSim)
        r = SceneRunner(s)
        t = 0.0
        for _ in range(25):
            t += w.dt
            r.step(w.dt, w.states(t), w.opts)
        out.append(s.save_state())
    for x, y in zip(out[0], out[1]):
        assert same(x, y)


@pytest.mark.parametrize("n,steps,cap", [(128, 20, 500_000), (256, 6, 4_000_000)])
def test_large_tank_invariants(n, steps, cap):
    """128^3 (about 4.7M particles) and the benchmark's 256^3 tank (about 38.6M) with the air field, drips, whitewater
    and the narrow band at full depth, no oracle: properties that hold at any size."""
    from splashtank_b200 import scenes
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = scenes.WaveTank(n, spray_cap=cap)
    s = w.make(FlipSim)
    r = SceneRunner(s)
    t = 0.0
    for _ in range(steps):
        t += w.dt
        r.step(w.dt, w.states(t), w.opts)
    st = s.readStats()
    p, v, ids = s.save_state()
    assert np.array_equal(np.sort(ids), np.arange(len(ids)))         # ids stay a permutation
    live = p[:, 1] >= -1e5
    assert int(live.sum()) >= len(w.pos) and np.isfinite(p[live]).all() and np.isfinite(v[live]).all()
    g = s.grid()
    # the cell counts (taken from the positions at the start of the step) cover every particle live at that time
    assert int(g["cnt"].sum()) == st["live"]
    assert (g["ctype"] & 255 == 1).sum() == st["fluid"]


@pytest.mark.parametrize("scene", ["dam", "tank"])
def test_pbf_density_stage(scene):
    """PBF density constraints (4 iterations) on the FLIP particles at the end of every step: a dam break thrown at a
    moving sphere (collider response after each correction, the sphere's boundary density), and the wave tank with
    whitewater, the air field and a 3-cell narrow band (refilled particles join the constraint): 20 steps bit for bit."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    from splashtank_b200.scene import SceneRunner, sphere_sdf
    if scene == "dam":
        sc = scenes.dam_break(32)
        sc["vel"] = np.tile(np.array([[1.5, 0.0, 0.0]], np.float32), (len(sc["pos"]), 1))
        g, o = make_pair(sc)
        sdf = sphere_sdf(0.12, 1 / 64, sid=3)
        opts = dict(sc["opts"], pbf=4)
        runs, t = [SceneRunner(s) for s in (g, o)], 0.0
        for _ in range(20):
            t += sc["dt"]
            st = [dict(id=1, sdf=sdf, x=0.1 - 0.5 * t, y=0.15, z=0.0)]
            for r in runs:
                r.step(sc["dt"], st, opts)
        assert_same_state(g, o)
    else:
        w, g, o = _tank_pair(32, 3.0)
        w.opts = dict(w.opts, pbf=dict(iters=4))
        _run_tank(w, (g, o), 20)
        assert_same_state(g, o, spray=True)


def test_dam_break_64_as_benchmarked():
    """The plain dam break exactly as its configuration states it: 64^3 MAC grid (dx 1/64) in 8^3 blocks, solid walls,
    fluid where x < 0.4 and y < 0.6, 8 particles per cell with seeded jitter (505,856 particles), FLIP 0.97, gravity
    9.81, dt 1/240, 50 red-black SOR iterations at omega 1.7, 100 steps: bit for bit with the oracle."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    sc = scenes.dam_break(64)
    assert len(sc["pos"]) == 505_856 and sc["opts"]["iters"] == 50 and sc["opts"]["omega"] == 1.7 and sc["steps"] == 100
    g, o = make_pair(sc, extra=0)
    o.set_threads(os.cpu_count() or 8)
    for _ in range(sc["steps"]):
        for s in (g, o):
            s.step(sc["dt"], sc["opts"])
    assert_same_state(g, o)


def _big_tank_pair(n, spray_cap):
    from oracle.oracle import OracleFlipSim
    from splashtank_b200 import scenes
    from splashtank_b200.flip import FlipSim
    w = scenes.WaveTank(n, spray_cap=spray_cap)
    g = w.make(FlipSim)
    o = w.make(OracleFlipSim, threads=os.cpu_count() or 8)
    return w, g, o


@pytest.mark.parametrize("n,steps,cap", [(128, 10, 500_000), (256, 3, 4_000_000)])
def test_wave_tank_at_benchmark_sizes(n, steps, cap):
    """The full-feature wave tank at 128^3 (about 4.7M particles, 10 steps) and at the benchmark's 256^3 (about 38.6M
    particles, 3 steps): piston and sphere colliders, narrow band at full depth with refills, whitewater, air field,
    drips, gusts and sheet tearing, every field bit for bit with the oracle (tile counts and particle indices at the
    benchmark's scale)."""
    w, g, o = _big_tank_pair(n, cap)
    _run_tank(w, (g, o), steps)
    assert g.readStats()["live"] > 0.9 * len(w.pos)
    assert_same_state(g, o, spray=True)
    g.destroy()
    o.destroy()


def test_empty_and_bad_arguments():
    import ctypes as C
    from splashtank_b200 import abi
    from splashtank_b200.flip import FlipSim, StError, load_library
    s = FlipSim(1 / 64, 1000, size=(1, 1, 1))
    s.step(1 / 240, dict(g=9.81, iters=4))                        # no particles: nothing happens
    assert s.readStats()["steps"] == 0
    f = load_library()[1]
    o = abi.default_opts()
    o.size = 3                                                      # wrong struct size
    assert f["flip_step"](s._h, 1 / 240, C.byref(o)) == abi.ST_BAD_ARG
    d = abi.FlipDesc()
    d.size = C.sizeof(abi.FlipDesc)
    d.d = -1.0
    h = C.c_void_p()
    assert f["flip_create"](C.byref(d), C.byref(h)) == abi.ST_BAD_ARG


def test_spray_pool_resized_mid_run_and_ring_recycling():
    """setSprayCap between steps (a smaller pool, then none, then one again: the slot counter keeps counting, the pool
    starts empty, the first pool brings the air field) and recycle off (add takes no more once the cap is reached)."""
    from flip_compare import make_pair
    from splashtank_b200 import scenes
    sc = scenes.dam_break(32)
    sc["vel"] = np.tile(np.array([[2.5, 0.5, 0.0]], np.float32), (len(sc["pos"]), 1))
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY, min=0.5), air=dict(on=True, couple=3.0, decay=0.6), gust=1.0)
    g, o = make_pair(sc, spray_cap=0)
    for s in (g, o):
        p, v, i = s.save_state()
        s.load_state(p, v, i, t=0.6, seed=0)
    for cap, steps in ((20000, 10), (3000, 10), (0, 3), (8000, 10)):
        for s in (g, o):
            s.setSprayCap(cap)
        for _ in range(steps):
            for s in (g, o):
                s.step(sc["dt"], opts)
        assert_same_state(g, o, spray=cap > 0)
    assert g.readStats()["spray_used"] > 8000
    for s in (g, o):
        s.recycle = False
        s.setCap(s.N)
    extra = np.zeros((5, 3), np.float32)
    assert g.add_many(extra) == o.add_many(extra) == 0
