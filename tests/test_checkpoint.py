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
    sp = sim.readSpray()
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
