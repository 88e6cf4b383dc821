"""Frames and bake measurements: st_flip_read_frame against the restatement of packFrameBuf (bit for bit),
st_flip_bake_diag against bakeDiag, the bake loop and the SPLC cache round trip."""
import numpy as np
import pytest

from splashtank_b200 import bake, scenes


def test_cache_round_trip():
    rng = np.random.default_rng(3)
    frames = []
    for k in range(4):
        n = int(rng.integers(0, 50))
        fr = dict(n=n, pos=rng.integers(0, 65536, (n, 3)).astype(np.uint16), spd=rng.integers(0, 256, n).astype(np.uint8),
                  fm=rng.integers(0, 256, n).astype(np.uint8) if k % 2 else None, objs=rng.random(12).astype(np.float32))
        frames.append(fr)
    meta = dict(d=0.01, fps=30, ids=[1, 2], b=dict(x0=-0.5, x1=0.5), engine="flip")
    buf = bake.write_cache(frames, meta)
    assert len(buf) % 4 == 0
    m2, f2 = bake.parse_cache(buf)
    assert m2 == meta and len(f2) == 4
    for a, b in zip(frames, f2):
        assert a["n"] == b["n"] and np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["spd"], b["spd"])
        assert (a["fm"] is None) == (b["fm"] is None) and (a["fm"] is None or np.array_equal(a["fm"], b["fm"]))
        assert np.array_equal(a["objs"], b["objs"])


def test_frame_checker_follows_the_javascript_arithmetic():
    from oracle.frames import pack_frame_buf
    box = (-0.5, 0.0, -0.5, 0.5, 1.0, 0.5)
    k = 65535.0
    buf = np.array([[-0.5 + 2.5 / k, 0.5, 0.0, 3.0 + 64 * 2], [0.0, -1e6, 0.0, 0.0], [0.25, 1.2, 0.0, 70.0], [0.0, -2e6, 0.0, 0.0]], np.float32)
    fr = pack_frame_buf(buf, 4, box, 1.0)
    assert fr["n"] == 3                                   # cut after the last live point
    assert fr["spd"][1] == 255 and tuple(fr["pos"][1]) == (0, 0, 0)
    assert fr["spd"][0] == 48 and fr["fm"][0] == 34       # speed 3 x 16, level 2 x 17
    assert fr["pos"][2][1] == 65535                       # clamped
    assert fr["spd"][2] == 96 and fr["fm"][2] == 17


@pytest.mark.gpu
def test_device_frame_and_diag_match_the_reference_arithmetic():
    from oracle.frames import bake_diag, pack_frame_buf
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=100_000)
    sim = tank.make(FlipSim)
    run = SceneRunner(sim)
    t = 0.0
    for _ in range(40):
        t += tank.dt
        run.step(tank.dt, tank.states(t), tank.opts)
    b = sim.b   # this tank's box bounds are exact in single precision (0, +-0.5, 1)
    box = (b["x0"], b["y0"], b["z0"], b["x1"], b["y1"], b["z1"])
    n = sim.N
    dst = np.zeros((n, 4), np.float32)
    sim.readbackInto(dst)
    for vs in (1.0, 1.7):
        got = sim.read_frame(vs)
        want = pack_frame_buf(dst, n, box, vs)
        assert got["n"] == want["n"] > 0
        assert np.array_equal(got["pos"], want["pos"]) and np.array_equal(got["spd"], want["spd"])
        assert (got["fm"] is None) == (want["fm"] is None)
        if got["fm"] is not None:
            assert np.array_equal(got["fm"], want["fm"])
    d = sim.bake_diag(tank.opts["vmax"])
    w = bake_diag(dst, n, box, tank.opts["vmax"])
    for key in ("alive", "gone", "nonFinite", "outsideBox", "atWaterSpeedLimit", "foamyPoints", "heightHist", "bbox"):
        assert d[key] == w[key], key
    for key in ("meanSpeed", "maxSpeed", "meanFoam"):
        assert abs(d[key] - w[key]) <= 1e-12 * max(1.0, abs(w[key])), key
    assert np.allclose(d["center"], w["center"], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_bake_loop_writes_a_cache():
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=0)
    sim = tank.make(FlipSim)
    run = SceneRunner(sim)
    par = dict(tank.opts)
    par.pop("spr", None)
    frames = bake.run_bake(sim, run, tank.states, par, fps=60, frames=4, substeps=2)
    assert len(frames) == 5 and all(d["sub"] >= 2 for _, d in frames[1:])
    assert frames[0][1]["alive"] == len(tank.pos)
    buf = bake.write_cache([f for f, _ in frames], dict(d=tank.d, fps=60, ids=[1, 2], engine="flip"))
    meta, back = bake.parse_cache(buf)
    assert len(back) == 5 and back[-1]["n"] == frames[-1][0]["n"] and np.array_equal(back[-1]["pos"], frames[-1][0]["pos"])
