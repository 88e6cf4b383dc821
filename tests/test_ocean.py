"""The ocean boundary (src/flip/wgsl-core.js:201-226 and its uses in classify, normFaces, g2p, the narrow band and the
whitewater; oceanWaves, src/shared.js:760-780).

CPU: the wave list against the dispersion relation and the spectrum's significant height, the product's host
computation equal to the oracle's; an ocean tank on the oracle (the boundary is a wall under the waves, particles that
drift into it are removed, nothing blows up). GPU: the same tank stepped by the device equals the oracle bit for bit."""
import ctypes as C
import os

import numpy as np
import pytest

from splashtank_b200 import scenes

OCEAN = dict(on=True, level=0.3, layer=0.12, length=0.35, height=0.05, dir=30.0, spread=20.0, seed=3)


def test_wave_list_follows_the_dispersion_relation():
    from splashtank_b200.flip import ocean_waves
    w = ocean_waves(OCEAN, 9.81).astype(np.float64)
    assert w.shape == (24, 8)
    k, om = w[:, 5], w[:, 3]
    np.testing.assert_allclose(om ** 2, 9.81 * k * np.tanh(k * 0.3), rtol=1e-5)          # omega^2 = g k tanh(k D)
    np.testing.assert_allclose(np.hypot(w[:, 0], w[:, 1]), k, rtol=1e-6)                   # (kx, kz) has length k
    hs = 4 * np.sqrt(np.sum(w[:, 2] ** 2) / 2)                                             # 4 standard deviations
    assert abs(hs - 0.05) < 0.005 and np.all(w[:, 2] <= 0.3 / k + 1e-7)
    ang = np.degrees(np.arctan2(w[:, 1], w[:, 0]))
    assert np.all(np.abs(ang - 30.0) <= 20.0 + 1e-3)                                      # within the spread
    assert ocean_waves(dict(OCEAN, height=0.0), 9.81)[:, 2].max() == 0.0


def test_host_wave_list_equals_the_oracle():
    from oracle.oracle import funcs
    from splashtank_b200 import abi
    from splashtank_b200.flip import make_opts, ocean_waves
    funcs()   # builds the oracle library when it is missing
    lib = C.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "liboracle_flip.so"))
    f = lib.oracle_ocean_waves
    f.argtypes, f.restype = [C.POINTER(abi.StepOpts), C.c_double, abi.f32p], C.c_int
    for oc in (OCEAN, dict(OCEAN, seed=0, dir=-75.0, spread=0.0, length=1.3), dict(OCEAN, height=0.4, length=0.08)):
        s, keep = make_opts(dict(g=9.81, ocean=oc))
        want = np.zeros(256, np.float32)
        n = f(C.byref(s), oc["level"], want.ctypes.data_as(abi.f32p))
        assert np.array_equal(ocean_waves(oc, 9.81).ravel(), want[:n * 8])


def ocean_pair(n=32, gpu=True):
    from oracle.oracle import OracleFlipSim
    sc = scenes.ocean_tank(n)
    sims = []
    classes = [OracleFlipSim]
    if gpu:
        from splashtank_b200.flip import FlipSim
        classes = [FlipSim, OracleFlipSim]
    for cls in classes:
        kw = dict(threads=8) if cls is OracleFlipSim else {}
        s = cls(sc["d"], len(sc["pos"]) + sc["spare"], size=sc["size"], ratio=sc["ratio"], spray_cap=sc["spray_cap"], **kw)
        s.add_many(sc["pos"], sc["vel"])
        park = np.zeros((sc["spare"], 3), np.float32)
        park[:, 1] = -1.0e6
        s.add_many(park)
        s.nb_fills(boxes=[], mode=1)
        sims.append(s)
    return sc, sims


def run(sc, sims, steps):
    t = 0.0
    for _ in range(steps):
        t += sc["dt"]
        for s in sims:
            s.step(sc["dt"], dict(sc["opts"], time=t))


def test_ocean_tank_on_the_oracle():
    sc, (o,) = ocean_pair(24, gpu=False)
    run(sc, [o], 20)
    p, v, _ = o.save_state()
    alive = p[:, 1] > -1e5
    assert np.isfinite(p[alive]).all() and np.abs(v[alive, :3]).max() < 2.0
    h = 1.0 / 24
    x, z = p[alive, 0] + 0.5, p[alive, 2] + 0.5
    lw = 1.0 - np.minimum(np.minimum(x, 1 - x), np.minimum(z, 1 - z)) / OCEAN["layer"]
    assert (lw < 0.5 + 2 * h / OCEAN["layer"]).all()              # no particle stays deep in the boundary
    G = o.grid()
    ty = (G["ctype"] & 0xff).reshape(o.tz * 8, o.ty * 8, o.tx * 8)
    # the boundary (cell centres within 0.06 of a side wall: the first column at h = 1/24) is a wall under the waves
    # (levels below 0.25 here) and air above them (above 0.35)
    assert (ty[:24, :6, 0] == 2).all() and (ty[:24, 9:20, 0] == 0).all() and (ty[1:23, :6, 1] != 2).all()


@pytest.mark.gpu
def test_device_ocean_tank_matches_the_oracle():
    """32^3 ocean tank, narrow band of 3 cells, whitewater and the air field, 40 steps: bit-exact."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_flip_parity import assert_same_state
    sc, (g, o) = ocean_pair(32)
    run(sc, (g, o), 40)
    assert_same_state(g, o, spray=True)
