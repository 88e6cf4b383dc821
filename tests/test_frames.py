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


def test_cache_round_trip_with_whitewater_and_deep_water():
    rng = np.random.default_rng(5)
    frames = []
    for k in range(3):
        n, ns, nd = int(rng.integers(1, 40)), int(rng.integers(0, 9)), int(rng.integers(0, 7))
        fr = dict(n=n, pos=rng.integers(0, 65536, (n, 3)).astype(np.uint16), spd=rng.integers(0, 256, n).astype(np.uint8), fm=None,
                  objs=np.zeros(0, np.float32),
                  sp=dict(n=ns, pos=rng.integers(0, 65536, (ns, 3)).astype(np.uint16), pk=rng.integers(0, 2 ** 32, ns, dtype=np.uint64).astype(np.uint32)),
                  dp=dict(n=nd, pos=rng.integers(0, 65536, (nd, 3)).astype(np.uint16), spd=rng.integers(0, 192, nd).astype(np.uint8)))
        frames.append(fr)
    buf = bake.write_cache(frames, dict(ids=[]))
    assert len(buf) % 4 == 0
    _, f2 = bake.parse_cache(buf)
    for a, b in zip(frames, f2):
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["spd"], b["spd"])
        for part, keys in (("sp", ("pos", "pk")), ("dp", ("pos", "spd"))):
            if a[part]["n"]:
                assert b[part]["n"] == a[part]["n"] and all(np.array_equal(a[part][k], b[part][k]) for k in keys)
            else:
                assert part not in b


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
def test_async_frame_matches_the_synchronous_one():
    """st_flip_read_frame_async: the frame of the particles at the call lands while later steps run and equals the
    synchronous frame taken at the same point; a second call first settles the pending one; a wait with nothing
    pending gives no points."""
    import torch
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=100_000)
    sim = tank.make(FlipSim)
    run = SceneRunner(sim)
    t = [0.0]

    def advance(k):
        for _ in range(k):
            t[0] += tank.dt
            run.step(tank.dt, tank.states(t[0]), tank.opts)

    def same(a, b):
        assert a["n"] == b["n"] > 0
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["spd"], b["spd"])
        assert (a["fm"] is None) == (b["fm"] is None)
        assert a["fm"] is None or np.array_equal(a["fm"], b["fm"])

    advance(30)
    assert sim.frame_wait()["n"] == 0
    cap = sim.MAXN
    pin = torch.empty(cap * 8, dtype=torch.uint8, pin_memory=True).numpy()
    out = (pin[:cap * 6].view(np.uint16).reshape(cap, 3), pin[cap * 6:cap * 7], pin[cap * 7:cap * 8])
    want = sim.read_frame(1.3)
    sim.read_frame_async(1.3, out=out)
    advance(3)   # steps queued behind the frame's packing while its copy runs
    same(sim.frame_wait(), want)
    assert sim.frame_wait()["n"] == 0
    want = sim.read_frame(1.0)
    sim.read_frame_async(1.0)
    sim.read_frame_async(1.0, out=out)
    same(sim.frame_wait(), want)
    advance(1)
    assert not np.array_equal(sim.read_frame(1.0)["pos"], want["pos"])


@pytest.mark.gpu
def test_async_stats_match_the_synchronous_ones():
    """st_flip_stats_async / st_flip_stats_wait: the counters of each step, read later, equal those read right after it
    on an identical tank; only the last four tickets are held."""
    from splashtank_b200.flip import FlipSim, StError
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=100_000)
    a, b = tank.make(FlipSim), tank.make(FlipSim)
    ra, rb = SceneRunner(a), SceneRunner(b)
    want, tickets = [], []
    t = 0.0
    for _ in range(6):
        t += tank.dt
        ra.step(tank.dt, tank.states(t), tank.opts)
        want.append(dict(a.readStats()))
        rb.step(tank.dt, tank.states(t), tank.opts)
        tickets.append(b.readStatsAsync())
    assert tickets == [1, 2, 3, 4, 5, 6]
    for k in range(2, 6):
        assert b.statsWait(tickets[k]) == want[k], k
    assert b.statsWait(tickets[5]) == want[5]   # a ticket can be read again while it is held
    for k in (0, 1):
        with pytest.raises(StError):
            b.statsWait(tickets[k])
    assert want[5]["steps"] == 6 and want[5]["live"] > 0


@pytest.mark.gpu
def test_track_reports_step_times():
    """track (src/gpu.js:444-454): once the queued steps have finished none is in flight, lastMs is the median of the
    recent step times and slowMs the largest, and the median is near the device time the stage timer measures."""
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=20_000)
    sim = tank.make(FlipSim)
    run = SceneRunner(sim)
    sim.track()
    assert sim.inflight == 0 and sim.lastMs == 0.0 and sim.slowMs == 0.0
    t = 0.0
    for _ in range(12):
        t += tank.dt
        run.step(tank.dt, tank.states(t), tank.opts)
    sim.readStats()   # waits for the stream
    sim.track()
    assert sim.inflight == 0
    assert 0.0 < sim.lastMs <= sim.slowMs < 1000.0
    timed = sim.stepTimed(tank.dt, dict(tank.opts, cols=[]))
    sim.track()
    assert sim.inflight == 0 and sim.lastMs < 5.0 * max(timed["total"], 0.05)


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


@pytest.mark.gpu
def test_bake_loop_stores_whitewater_and_deep_water():
    """With a whitewater pool and the deep look (narrow band of 3 cells), every frame after the first carries the
    whitewater and deep-water parts, and the cache keeps them."""
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    tank = scenes.WaveTank(32, steps=60, spray_cap=20000, band=3.0)
    sim = tank.make(FlipSim)
    frames = bake.run_bake(sim, SceneRunner(sim), tank.states, dict(tank.opts), fps=60, frames=3, substeps=2, nb_look=True)
    last, diag = frames[-1]
    assert last["dp"]["n"] > 100 and diag["deepPoints"] == last["dp"]["n"] and "sprayPoints" in diag
    buf = bake.write_cache([f for f, _ in frames], dict(d=tank.d, fps=60, ids=[1, 2], engine="flip"))
    _, back = bake.parse_cache(buf)
    assert back[-1]["dp"]["n"] == last["dp"]["n"] and np.array_equal(back[-1]["dp"]["pos"], last["dp"]["pos"])


def test_spray_codes_follow_the_javascript_arithmetic():
    """packSprayJS (src/flip/bake.js:4-15), worked by hand: speed in quarter units from bit 21, kind bits, octahedral
    direction (Math.round: 511.5 rounds up to 512) or the foam's life left."""
    from oracle.frames import pack_spray_js
    v = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, -2.0], [0.0, 3.0, 0.0]])
    got = pack_spray_js(v, np.array([0.0, 0.0, 1.0, 2.0]), np.array([0.5, 0.5, 0.5, 0.25]))
    want = [0x80000000 | (1023 << 10) | 512,                       # at rest: straight up
            0x80000000 | (4 << 21) | (512 << 10) | 1023,            # +x at speed 1
            0x80000000 | (8 << 21) | 0x40000000 | (1023 << 10) | 1023,   # mist falling -z: folded octahedron
            0x80000000 | (12 << 21) | 0x20000000 | 256]             # foam with a quarter of its life left (255.75 -> 256)
    assert [int(x) for x in got] == want


def test_deep_points_pack_like_pack_deep():
    from oracle.frames import pack_deep
    box = (-0.5, 0.0, -0.5, 0.5, 1.0, 0.5)
    d = pack_deep(np.array([[0.0, 0.5, 0.0, 4096.0 + 2.5], [0.0, -1e6, 0.0, 0.0], [0.5, 1.0, -0.5, 4096.0 + 63.0]], np.float32), box, 1.0)
    assert d["n"] == 2                                         # the gone point is left out
    assert tuple(d["pos"][0]) == (32768, 32768, 32768) and d["spd"][0] == 40
    assert tuple(d["pos"][1]) == (65535, 65535, 0) and d["spd"][1] == 191


def _spray_scene():
    from flip_compare import make_pair
    sc = scenes.dam_break(32)
    sc["vel"] = np.tile(np.array([[2.5, 0.5, 0.0]], np.float32), (len(sc["pos"]), 1))
    opts = dict(sc["opts"], spr=dict(scenes.APP_SPRAY, min=0.5), gust=1.0, nb=dict(on=True, band=3.0))
    g, o = make_pair(sc, spray_cap=30000)
    for s in (g, o):
        p, v, i = s.save_state()
        s.load_state(p, v, i, t=0.6, seed=0)
    for _ in range(30):
        for s in (g, o):
            s.step(sc["dt"], opts)
    return g, o


@pytest.mark.gpu
def test_device_spray_frame_matches_pack_spray_frame():
    """The frame's whitewater part packed on the device equals packSprayFrame of the pool read back, with every
    living slot (cap above the living count) and with a sampling step (cap 500)."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle.frames import pack_spray_frame
    g, _ = _spray_scene()
    b = g.b
    box = (b["x0"], b["y0"], b["z0"], b["x1"], b["y1"], b["z1"])
    sd = g.readSpray()
    for cap in (200000, 500):
        got = g.read_spray_frame(cap, 3.0)
        want = pack_spray_frame(sd["p"], sd["v"], sd["n"], box, cap, 3.0)
        assert got["alive"] == want["alive"] > 500 and got["n"] == want["n"] > 0
        assert np.array_equal(got["pos"], want["pos"]) and np.array_equal(got["pk"], want["pk"])
    kinds = (g.read_spray_frame()["pk"] >> 29) & 3
    assert len(set(kinds.tolist())) == 4                      # spray, foam, mist and bubble codes all present


@pytest.mark.gpu
def test_device_deep_points_and_live_view_match_the_oracle():
    """Narrow band of 3 cells on a 96^3 tank (2.05M particle slots: the live view samples every 7th), deep look on:
    the deep water points and the packed live view equal the oracle's. About 240k deep cells: the first pass keeps the
    first 200,000, later passes a hashed sample sized by the previous count."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle.frames import pack_deep, pack_live
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = scenes.WaveTank(96, spray_cap=50000, band=3.0)
    g, o = w.make(FlipSim), w.make(OracleFlipSim, threads=8)
    for s in (g, o):
        s.setDeepLook(True)
    runs, t = [SceneRunner(s) for s in (g, o)], 0.0
    for _ in range(6):
        t += w.dt
        st = w.states(t)
        for r in runs:
            r.step(w.dt, st, w.opts)
    b = g.b
    box = (b["x0"], b["y0"], b["z0"], b["x1"], b["y1"], b["z1"])
    counts = []
    for vs in (1.0, 1.5):
        got, pts = g.read_deep(vs), o.deep_points()
        want = pack_deep(pts, box, vs)
        assert got["n"] == want["n"]
        assert np.array_equal(got["pos"], want["pos"]) and np.array_equal(got["spd"], want["spd"])
        counts.append(got["n"])
    assert counts[0] == 200000 and 190000 < counts[1] < 200000
    words, L = g.pack_live(1.2)
    assert L["from_pos"] == 0 and L["n_deep"] == 200000
    pos, _, _ = o.save_state()
    sd = o.readSpray()
    used = min(o.readStats()["spray_used"], o.sprayCap)
    stride = max(1, -(-o.N // 300000))
    assert stride == 7 and L["n_water"] == -(-o.N // stride)
    want = pack_live(L, pos, stride, sd["p"], sd["v"], used, min(o.sprayCap, 200000), 3.0, o.deep_points(), box, 1.2)
    assert words[1] == want[1] > 190000
    assert np.array_equal(words, want)


@pytest.mark.gpu
def test_device_live_view_with_whitewater_matches_the_oracle():
    """The live view of a tank full of whitewater (every kind): water, whitewater codes in the shader's f32 packSpray."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle.frames import pack_live
    g, o = _spray_scene()
    b = g.b
    box = (b["x0"], b["y0"], b["z0"], b["x1"], b["y1"], b["z1"])
    words, L = g.pack_live(1.0)
    assert L["from_pos"] == 0 and L["n_spray"] == 30000 and L["n_deep"] == 0
    pos, _, _ = o.save_state()
    sd = o.readSpray()
    used = min(o.readStats()["spray_used"], o.sprayCap)
    want = pack_live(L, pos, 1, sd["p"], sd["v"], used, 30000, 3.0, None, box, 1.0)
    assert words[0] == want[0] > 1000
    assert np.array_equal(words, want)


@pytest.mark.gpu
def test_read_deep_points_pump_and_mem_bytes():
    """readDeep's raw points equal the oracle's deep pass; pump() unpacks the packed live view into outFrame; memBytes
    counts what the handle holds, including the buffers its first frame and live view allocate."""
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = scenes.WaveTank(48, spray_cap=20000, band=3.0)
    g, o = w.make(FlipSim), w.make(OracleFlipSim, threads=8)
    m0 = g.memBytes()
    assert m0 > 48 ** 3 * 40
    for s in (g, o):
        s.setDeepLook(True)
    runs, t = [SceneRunner(s) for s in (g, o)], 0.0
    for _ in range(4):
        t += w.dt
        for r in runs:
            r.step(w.dt, w.states(t), w.opts)
    d = g.readDeep()
    want = o.deep_points()
    assert d["n"] == len(want) > 1000 and np.array_equal(d["p"], want)
    fr = g.pump(1.0)
    assert g.gen == 1 and fr["n"] == g.N and fr["dp"]["n"] > 1000 and fr["pos"].shape == (g.N, 3)
    assert g.memBytes() > m0
    g.read_frame()
    assert g.memBytes() >= m0 + g.MAXN * 8
