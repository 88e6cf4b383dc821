"""Full checkpoint (st_flip_save_full / st_flip_load_full): a restored tank continues bit-identically."""
import copy

import numpy as np
import pytest

from splashtank_b200 import scenes


def _state(sim):
    n = sim.N
    p = np.zeros((max(n, 1), 4), np.float32)
    v = np.zeros((max(n, 1), 4), np.float32)
    sim.readbackInto(p, v)
    sp = sim.readSpray() or {"p": np.zeros((0, 4), np.float32), "v": np.zeros((0, 4), np.float32)}   # None without a pool
    st = sim.readStats()
    return p[:n].copy(), v[:n].copy(), sp["p"].copy(), sp["v"].copy(), (st["live"], st["fluid"], st["sc"], st["spray_used"])


def _same(a, b):
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert a[4] == b[4]


@pytest.mark.gpu
def test_full_checkpoint_continues_bit_identically():
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=200_000)
    sim = tank.make(FlipSim)
    run = SceneRunner(sim)
    t = 0.0
    for _ in range(40):   # past 0.1 s, when whitewater emission starts
        t += tank.dt
        run.step(tank.dt, tank.states(t), tank.opts)
    blob = sim.save_full()
    prev, t_saved = copy.deepcopy(run.prev), t

    def go(s, r, t0):
        tt = t0
        for _ in range(5):
            tt += tank.dt
            r.step(tank.dt, tank.states(tt), tank.opts)
        return _state(s)
    a = go(sim, run, t_saved)
    # a fresh handle with the same geometry, restored
    sim2 = tank.make(FlipSim)
    sim2.load_full(blob)
    run2 = SceneRunner(sim2)
    run2.prev = copy.deepcopy(prev)
    b = go(sim2, run2, t_saved)
    _same(a, b)
    # the first handle, rewound
    sim.load_full(blob)
    run.prev = copy.deepcopy(prev)
    _same(a, go(sim, run, t_saved))
    assert a[4][3] > 0   # whitewater was emitted, so the ring round-trips too
    sim.destroy()
    sim2.destroy()


@pytest.mark.gpu
def test_full_checkpoint_rejects_another_geometry():
    from splashtank_b200.flip import FlipSim, StError
    a = scenes.WaveTank(32, steps=4, spray_cap=1000).make(FlipSim)
    b = scenes.WaveTank(40, steps=4, spray_cap=1000).make(FlipSim)
    with pytest.raises(StError, match="geometry"):
        b.load_full(a.save_full())


def _hdr_words(blob):
    """The checkpoint header's 32-bit words (magic, version, nx, ny, nz, ntiles, ncell, maxN, sprayCap, N, cap, ring, ...)."""
    return np.frombuffer(blob, np.uint32, count=24).copy()


def _patched(blob, word, value):
    b = bytearray(blob)
    b[word * 4:word * 4 + 4] = np.uint32(value).tobytes()
    return bytes(b)


@pytest.mark.gpu
def test_full_checkpoint_rejects_tampered_or_short_blobs_and_keeps_the_tank():
    """Counters out of range (cap above the capacity, N above cap, ring at or past cap) and a truncated blob are
    rejected before anything of the handle changes: the tank then steps exactly as one that was never given them."""
    from splashtank_b200.flip import FlipSim, StError
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=20, spray_cap=20_000)
    a, b = tank.make(FlipSim), tank.make(FlipSim)
    ra, rb = SceneRunner(a), SceneRunner(b)
    t = 0.0
    for _ in range(6):
        t += tank.dt
        for r in (ra, rb):
            r.step(tank.dt, tank.states(t), tank.opts)
    blob = a.save_full()
    w = _hdr_words(blob)
    maxN, N, cap = int(w[7]), int(w[9]), int(w[10])
    bad = [_patched(blob, 10, maxN + 1), _patched(blob, 9, cap + 1), _patched(blob, 11, cap), blob[:len(blob) - 4096], blob[:200]]
    for x in bad:
        with pytest.raises(StError):
            b.load_full(x)
    assert b.N == N
    for _ in range(4):
        t += tank.dt
        for r in (ra, rb):
            r.step(tank.dt, tank.states(t), tank.opts)
    _same(_state(a), _state(b))
    a.destroy()
    b.destroy()


@pytest.mark.gpu
def test_full_checkpoint_carries_a_pending_fill_volume_restart():
    """A checkpoint taken while a narrow-band restart with a water-mesh fill volume is pending: the restored handle's
    first step starts the depth field from the same fill volume, so both continue bit for bit."""
    from test_oracle import shell_drop
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import sphere_sdf
    r, c = 0.22, (0.0, 0.45, 0.0)
    a, opts = shell_drop(FlipSim, r=r, c=c)
    b, _ = shell_drop(FlipSim, r=r, c=c)
    for _ in range(2):
        a.step(1.0 / 240.0, opts)
    a.nb_fill_vols([dict(sdf=sphere_sdf(r, a.h / 2, sid=9), x=c[0], y=c[1], z=c[2])])
    a.nb_fills(boxes=[(-0.5, 0.0, -0.5, 0.5, 0.05, 0.5)], mode=2)
    b.load_full(a.save_full())
    for _ in range(3):
        for s in (a, b):
            s.step(1.0 / 240.0, opts)
    _same(_state(a), _state(b))
    ga, gb = a.grid(), b.grid()
    assert np.array_equal(ga["ctype"], gb["ctype"])
