"""CPU tests of the oracle (oracle/flip_oracle.cpp): invariants of the reference step, a hydrostatic known answer,
the canonical storage order, edge cases (empty, open faces, ring recycling), and the committed golden fixtures."""
import os
import sys

import numpy as np
import pytest

from oracle.oracle import OracleFlipSim
from splashtank_b200 import scenes
from splashtank_b200.scene import SceneRunner

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def dam(n=16, extra=0, **kw):
    sc = scenes.dam_break(n)
    s = OracleFlipSim(sc["d"], len(sc["pos"]) + extra, size=sc["size"], ratio=sc["ratio"], threads=4, **kw)
    s.add_many(sc["pos"], sc["vel"])
    return s, sc


def cell_keys(s, p):
    """storage key of the cell of each position (tile-major, 512 cells per tile, x fastest inside)"""
    g = np.floor((p[:, :3].astype(np.float32) - np.array([s.b["x0"], s.b["y0"], s.b["z0"]], np.float32)) * np.float32(1.0 / s.h))
    i = np.clip(g[:, 0].astype(np.int64), 0, s.nx - 1)
    j = np.clip(g[:, 1].astype(np.int64), 0, s.ny - 1)
    k = np.clip(g[:, 2].astype(np.int64), 0, s.nz - 1)
    t = (i >> 3) + s.tx * ((j >> 3) + s.ty * (k >> 3))
    return t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7))


def test_empty_step_is_not_ready():
    s = OracleFlipSim(1 / 32, 100, size=(1, 1, 1), threads=1)
    s.step(1 / 240, dict(g=9.81, iters=5))   # returns early like FlipSim.step with N == 0 (src/flip/sim.js:181)
    assert s.readStats()["steps"] == 0


def test_invariants_after_steps():
    s, sc = dam(16)
    for _ in range(12):
        s.step(sc["dt"], sc["opts"])
    st = s.readStats()
    p, v = s.particles()
    assert st["live"] == len(sc["pos"]) == st["n"]            # closed box: nothing is lost
    m = 0.3 * s.d
    assert (p[:, 0] >= s.b["x0"] + m - 1e-6).all() and (p[:, 0] <= s.b["x1"] - m + 1e-6).all()
    assert (p[:, 1] >= s.b["y0"] + m - 1e-6).all() and (p[:, 1] <= s.b["y1"] - m + 1e-6).all()
    g = s.grid()
    assert g["cnt"].sum() == st["live"]                       # every live particle counted once
    keys = cell_keys(s, p)
    tiles = keys // 512
    assert g["tile_on"][tiles].all()                          # each particle's tile has storage
    assert (g["ctype"] & 255 == 1).sum() == st["fluid"]
    assert np.isfinite(p).all() and np.isfinite(v).all()


def test_storage_order_is_cell_then_id():
    s, sc = dam(16)
    for _ in range(3):
        s.step(sc["dt"], sc["opts"])
    # the order a step sorts into is defined by the positions at the start of that step: replay one step from a saved state
    p0, v0, i0 = s.save_state()
    s.step(sc["dt"], sc["opts"])
    _, _, i1 = s.save_state()
    k = cell_keys(s, p0)
    want = i0[np.lexsort((i0, k))]
    assert np.array_equal(i1, want)


def test_hydrostatic_pressure_known_answer():
    """Still water: after projection the vertical face velocity is 0, so the pressure rises by g*h per cell of depth."""
    n = 16
    h = 1.0 / n
    rng = np.random.default_rng(3)
    cells = scenes.box_cells((n, n, n), lambda ci, cj, ck: cj * h < 0.5)
    pos = scenes.seed_cells(cells, h, rng, -0.5, 0.0, -0.5)
    s = OracleFlipSim(h / 2, len(pos), size=(1, 1, 1), threads=4)
    s.add_many(pos)
    o = dict(g=9.81, flip=0.97, iters=400, omega=1.7, comp=0.0)
    for _ in range(6):
        s.step(1 / 240, o)
    g = s.grid()
    pres = g["pres"][:n, :n, :n]
    col = pres[n // 2, :, :].mean(axis=1)                     # rows j (depth profile) at mid z
    dp = -np.diff(col[2:6])                                   # pressure drop per cell going up, well inside the water
    assert np.allclose(dp, 9.81 * h, rtol=0.15), (dp, 9.81 * h)


def test_open_face_kills_and_dead_go_last():
    s, sc = dam(16, open=4)                                   # open floor: water falls out
    for _ in range(40):
        s.step(sc["dt"], sc["opts"])
    st = s.readStats()
    assert st["live"] < st["n"]
    p0, v0, i0 = s.save_state()
    dead0 = p0[:, 1] < -1e5
    assert (v0[dead0] == 0).all()
    s.step(sc["dt"], sc["opts"])                              # the sort at the start of a step moves the dead last
    p1, v1, i1 = s.save_state()
    nd = int(dead0.sum())
    assert np.array_equal(i1[len(i1) - nd:], i0[dead0])       # in their previous relative order
    assert (p1[len(p1) - nd:, 1] < -1e5).all()


def test_ring_recycles_slots_when_full():
    s = OracleFlipSim(1 / 32, 10, size=(1, 1, 1), threads=1)
    pts = np.array([[0.1 * k - 0.4, 0.2, 0.0] for k in range(13)], np.float32)
    assert s.add_many(pts) == 13                              # the last 3 overwrite slots 0..2 (src/gpu.js:390-394)
    assert s.readStats()["n"] == 10
    p, _, ids = s.save_state()
    assert np.allclose(p[:3, 0], pts[10:, 0]) and np.array_equal(ids, np.arange(10))


def test_narrow_band_full_depth_keeps_particles():
    w = scenes.WaveTank(24, spray_cap=20000)
    s = w.make(OracleFlipSim, threads=4)
    r = SceneRunner(s)
    t = 0.0
    n0 = len(w.pos)
    for _ in range(10):
        t += w.dt
        r.step(w.dt, w.states(t), w.opts)
    st = s.readStats()
    assert st["live"] >= n0                                   # full depth trims nothing; refills may add
    g = s.grid()
    phi = 8.0 - (g["ctype"] >> 16) / 4096.0
    deep = (g["ctype"] & 255) == 1
    assert (phi[deep] < 0.5).mean() > 0.9                     # water cells carry a negative depth


def shell_drop(cls, n=24, r=0.22, c=(0.0, 0.45, 0.0), band=3.0, seed=4, **kw):
    """A ball of water with particles only in the narrow band under its surface (nbSeed's 'vol' and sphere branches,
    src/shared.js:806-847, with seeded jitter): the tank, the particles and the step options."""
    h = 1.0 / n
    rng = np.random.default_rng(seed)
    cells = scenes.box_cells((n, n, n), lambda ci, cj, ck: np.abs(np.sqrt((ci * h - 0.5 - c[0]) ** 2 + (cj * h - c[1]) ** 2 +
                                                                           (ck * h - 0.5 - c[2]) ** 2) - (r - 0.5 * band * h)) < 0.5 * band * h)
    pos = scenes.seed_cells(cells, h, rng, -0.5, 0.0, -0.5)
    s = cls(h / 2, len(pos) + 4000, size=(1.0, 1.0, 1.0), **kw)
    s.add_many(pos)
    opts = dict(g=9.81, flip=0.95, comp=6.0, iters=30, vmax=14.0, nb=dict(on=True, band=band))
    return s, opts


def test_fill_volume_starts_the_depth_field_like_its_shape():
    """A water mesh given as a fill volume (its distance grid, fillPhi's loop over the records after the colliders,
    wgsl-core.js:235) starts the depth field as the same ball given as a sphere fill does, to the grid's interpolation
    error; a restart consumes the fills, so a second restart without new ones starts from air."""
    from splashtank_b200.scene import sphere_sdf
    r, c = 0.22, (0.0, 0.45, 0.0)
    a, opts = shell_drop(OracleFlipSim, r=r, c=c, threads=4)
    b, _ = shell_drop(OracleFlipSim, r=r, c=c, threads=4)
    a.nb_fills(spheres=[(c[0], c[1], c[2], r)])
    b.nb_fill_vols([dict(sdf=sphere_sdf(r, a.h / 2, sid=9), x=c[0], y=c[1], z=c[2])])
    for s in (a, b):
        s.step(1.0 / 240.0, opts)
    phi = [8.0 - (s.grid()["ctype"] >> 16) / 4096.0 for s in (a, b)]
    on = a.grid()["tile_on"].astype(bool)
    assert np.array_equal(on, b.grid()["tile_on"].astype(bool))
    near = phi[0] < 1.0   # inside the ball and a cell around it, where the distance grid reaches
    assert near.sum() > 1000 and (phi[0][near] < 0).sum() > 500
    assert np.max(np.abs(phi[0][near] - phi[1][near])) < 0.05
    assert phi[1].min() < -4.0   # deeper than the particles alone make it (about -2.5 from a band of 3)
    st = [s.readStats() for s in (a, b)]
    assert st[0]["live"] == st[1]["live"] and st[0]["fluid"] > 0


def test_air_field_settles_to_the_wind():
    """With no coupling, every air cell relaxes towards the wind by 1 - exp(-decay dt) a step (airUpdate,
    src/flip/wgsl-whitewater.js:67-86); a uniform field stays uniform under the blur. The grid is airAlloc's
    (src/flip/sim.js:343-350): r = 2 solver cells at 16^3, so 8 + 1 cells per axis."""
    s, sc = dam(16, spray_cap=100)
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY), wind=(1.0, 0.0, -0.5), air=dict(on=True, couple=0.0, decay=0.6))
    assert s.read_air().shape == (9, 9, 9, 3) and not s.read_air().any()
    steps = 12
    for _ in range(steps):
        s.step(sc["dt"], opts)
    a = s.read_air().reshape(-1, 3)
    left = np.exp(-0.6 * sc["dt"]) ** steps
    np.testing.assert_allclose(a, np.tile([1.0 - left, 0.0, -0.5 * (1.0 - left)], (len(a), 1)), rtol=1e-4, atol=1e-6)
    s.step(sc["dt"], dict(opts, air=None))   # off: the field is kept as it is
    np.testing.assert_array_equal(s.read_air().reshape(-1, 3), a)
    s.clear()
    assert not s.read_air().any()


def test_air_field_follows_the_water():
    """Coupled to moving water, the air near the surface picks up the water's direction."""
    s, sc = dam(16, spray_cap=100)
    s2 = OracleFlipSim(sc["d"], len(sc["pos"]), size=sc["size"], ratio=sc["ratio"], threads=4, spray_cap=100)
    vel = np.tile(np.array([[1.5, 0.0, 0.0]], np.float32), (len(sc["pos"]), 1))
    s2.add_many(sc["pos"], vel)
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY), air=dict(on=True, couple=3.0, decay=0.6))
    for _ in range(10):
        s2.step(sc["dt"], opts)
    a = s2.read_air()
    assert a[..., 0].max() > 0.1 and a[..., 0].sum() > 0 and np.all(np.isfinite(a))


def _drip_run(steps, y_of_t, dry=3.0, rate=20.0):
    from splashtank_b200.scene import sphere_sdf
    s, sc = dam(16, spray_cap=2000)
    sdf = sphere_sdf(0.1, 0.01, sid=5)
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY, rate=0.0), drip=dict(on=True, rate=rate, dry=dry))
    r, t = SceneRunner(s), 0.0
    for _ in range(steps):
        t += sc["dt"]
        r.step(sc["dt"], [dict(id=1, sdf=sdf, x=-0.3, y=y_of_t(t), z=0.0)], opts)
    return s, sc


def test_drip_samples_lie_on_the_surface():
    """dripSamples (src/flip/bake.js:19-40): points of the distance grid near the surface moved onto it along the
    gradient, about one per solver cell of surface (4 pi r^2 / h^2 = 32 at h = 1/16, so the floor of 100 applies)."""
    s, _ = _drip_run(1, lambda t: 0.8)
    d = s.read_drips()
    assert len(d) == 100
    p, n = d[:, 0:3].astype(np.float64), d[:, 4:7].astype(np.float64)
    assert np.all(d[:, 3] == 0)                                          # collider number
    np.testing.assert_allclose(np.linalg.norm(p, axis=1), 0.1, atol=2e-3)   # on the sphere
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-5)
    assert np.min(np.sum(n * p, axis=1) / np.linalg.norm(p, axis=1)) > 0.99   # normals point out
    assert np.all(d[:, 7] == 0)                                          # out of the water from the start: dry


def test_drips_wet_in_water_then_dry_out():
    """A sphere held in the water is wet (1); lifted out, its wetness falls by dt / dry a step (dripStep,
    src/flip/wgsl-whitewater.js:254-278) and it lets go of drops, which fly as spray with twice the spray life."""
    s, sc = _drip_run(8, lambda t: 0.3)
    assert np.all(s.read_drips()[:, 7] == 1.0)                           # in the water everywhere
    s2, sc = _drip_run(8 + 30, lambda t: 0.3 if t < 8.5 * sc["dt"] else 0.9)
    w = s2.read_drips()[:, 7]
    assert np.all(w < 1.0) and np.all(w > 1.0 - 31 * sc["dt"] / 3.0)
    np.testing.assert_allclose(w.max(), 1.0 - 30 * sc["dt"] / 3.0, atol=1e-4)
    st, sp = s2.readStats(), s2.readSpray()
    assert st["spray_used"] > 0
    alive = sp["p"][:, 3] > 0
    assert np.all(sp["v"][alive, 3] < 0.5)                               # spray kind (the fraction is time held)


@pytest.mark.parametrize("name", ["dam_break_16_s10", "wave_tank_24_s8"])
def test_golden_fixture(name):
    """The oracle still produces the committed fixtures (tests/golden/make_golden.py) bit for bit."""
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    ref = np.load(path)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from golden.make_golden import run_case
    got = run_case(name)
    for k in ref.files:
        assert np.array_equal(np.asarray(got[k]).view(np.uint8), ref[k].view(np.uint8)), k
