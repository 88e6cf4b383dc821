"""FlipSim: the reference simulator's per-step API (src/flip/sim.js FlipSim) over the C ABI.

Method and field names follow the JavaScript class so callers (a scene runner, a bake loop, tests) read the
same: ``step(dt, o)``, ``add``, ``fillBox``, ``fillSphere``, ``readbackInto``, ``readSpray``, ``clear``,
``setCap``, ``stepTimed``, ``activeCells``, ``stats``, ``N``, ``MAXN``, ``h``, ``b``.  The options object
``o`` is a dict with the reference's keys (g, iters, flip, comp, omega, vmax, wind, drag, foamTau, foamSens,
gust, tear, vs, cols, spr, nb).

The compute runs in libsplashtank_cuda.so (hand-written sm_100a kernels).  There is no CPU fallback: if the
library or a GPU is missing, construction raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_LIB = None
_FUNCS = None


def lib_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsplashtank_cuda.so")


def load_library():
    """Load the CUDA library (raises OSError when it has not been built)."""
    global _LIB, _FUNCS
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise OSError("splashtank_b200: %s is missing; build it with `python -m splashtank_b200.build`" % path)
        lib = C.CDLL(path)
        funcs = abi.bind(lib, "st_", abi.FLIP_FUNCS + abi.CUDA_ONLY_FUNCS)
        _LIB, _FUNCS = lib, funcs
    return _LIB, _FUNCS


class StError(RuntimeError):
    pass


def status_error(what, st):
    """StError for a failed call: the status name and the library's last error text on this thread."""
    e = load_library()[1].get("last_error")
    t = e() if e else None
    msg = t.decode() if t else ""
    name = abi.STATUS_NAMES[st] if 0 <= st < len(abi.STATUS_NAMES) else str(st)
    return StError(("%s failed: %s %s" % (what, name, msg)).rstrip())


def _f32(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(abi.f32p)


class _ColliderPack:
    """Keeps the ctypes collider records and SDF blobs alive for one call."""

    def __init__(self, cols):
        self.sdfs, self.keep = {}, []
        n = len(cols)
        self.arr = (abi.Collider * max(n, 1))()
        for k, c in enumerate(cols):
            sd = c["sdf"]
            sid = int(sd["id"])
            if sid not in self.sdfs:
                data = np.ascontiguousarray(sd["data"], dtype=np.float32)
                s = abi.Sdf()
                s.id = sid
                s.dims[:] = [int(x) for x in sd["dims"]]
                s.origin[:] = [float(x) for x in sd["origin"]]
                s.cell = float(sd["cell"])
                s.data = data.ctypes.data_as(abi.f32p)
                self.keep.append(data)
                self.sdfs[sid] = s
            r = self.arr[k]
            r.sdf = C.pointer(self.sdfs[sid])
            r.pos[:] = [float(c.get("x", 0)), float(c.get("y", 0)), float(c.get("z", 0))]
            r.R[:] = [float(x) for x in c.get("R", (1, 0, 0, 0, 1, 0, 0, 0, 1))]
            r.vel[:] = [float(c.get("vx", 0)), float(c.get("vy", 0)), float(c.get("vz", 0))]
            r.ang[:] = [float(c.get("wx", 0)), float(c.get("wy", 0)), float(c.get("wz", 0))]
        self.n = n


def make_opts(o, opt=None, default=None):
    """The options object o (src/flip/sim.js:185-230) as an st_step_opts; returns (opts, keepalive)."""
    s = default if default is not None else abi.default_opts()
    opt = opt or {}
    s.g = float(o.get("g", 9.81))
    s.iters = int(opt.get("iters") or o.get("iters", 30))
    for key, field in (("flip", "flip"), ("comp", "comp"), ("omega", "omega"), ("vmax", "vmax"), ("drag", "drag"),
                       ("foamTau", "foam_tau"), ("foamSens", "foam_sens"), ("gust", "gust"), ("tear", "tear"), ("vs", "vs")):
        if o.get(key) is not None:
            setattr(s, field, float(o[key]))
    w = o.get("wind") or (0, 0, 0)
    s.wind[:] = [float(x) for x in w]
    flags = 0
    if opt.get("noFoam"):
        flags |= abi.ST_OPT_NO_FOAM
    if opt.get("noCull"):
        flags |= abi.ST_OPT_NO_CULL
    if opt.get("fastAir"):
        flags |= abi.ST_OPT_FAST_AIR
    s.flags = flags
    cols = _ColliderPack(o.get("cols") or [])
    s.ncols = cols.n
    s.cols = C.cast(cols.arr, C.POINTER(abi.Collider))
    sp = o.get("spr")
    s.spray_on = 1 if sp else 0
    if sp:
        for key in ("rate", "min", "life", "mist", "drag", "mdrag"):
            setattr(s.spray, key, float(sp.get(key, 0)))
        ww = sp.get("ww") or {}
        s.spray.foam_life = float(ww.get("foamLife") or 3.0)
        s.spray.rise = float(ww.get("rise") or 0.3)
        s.spray.crest = float(ww["crest"]) if ww.get("crest") is not None else 1.0
        s.spray.impact = float(ww["impact"]) if ww.get("impact") is not None else 0.5
    nb = o.get("nb")
    s.nb_on = 1 if (nb and nb.get("on")) else 0
    s.nb_band = float(max(2.0, (nb or {}).get("band") or 3.0))
    air = o.get("air")
    s.air_on = 1 if (air and air.get("on")) else 0
    s.air_couple = float((air or {}).get("couple", 0.0))
    s.air_decay = float((air or {}).get("decay", 0.0))
    s.air_blur = float((air or {}).get("blur", 0.35))
    drip = o.get("drip")
    s.drip_on = 1 if (drip and drip.get("on")) else 0
    s.drip_rate = float((drip or {}).get("rate", 0.0))
    s.drip_dry = float((drip or {}).get("dry", 1.0))
    oc = o.get("ocean")
    s.ocean_on = 1 if (oc and oc.get("on")) else 0
    if oc:
        s.ocean_level = float(oc.get("level", 0.0))
        s.ocean_layer = float(oc.get("layer", 0.0))
        s.ocean_length = float(oc.get("length", 0.0))
        s.ocean_height = float(oc.get("height", 0.0))
        s.ocean_dir = float(oc.get("dir", 0.0))
        s.ocean_spread = float(oc.get("spread", 0.0))
        s.ocean_seed = int(oc.get("seed", 0))
    s.time = float(o.get("time") or 0.0)
    # PBF density constraints on the particles after g2p: o.pbf = iterations, or {"iters": n}
    pb = o.get("pbf")
    s.pbf_iters = int((pb.get("iters", 0) if isinstance(pb, dict) else pb) or 0)
    return s, cols


def ocean_waves(ocean, g=9.81, depth=None, y0=0.0):
    """oceanWaves (src/shared.js:760-780) through st_ocean_waves: (24, 8) float32 rows kx, kz, amplitude, angular
    frequency, phase, wavenumber, 0, 0. depth defaults to the mean level above y0."""
    s, keep = make_opts(dict(g=g, ocean=dict(ocean, on=True)))
    w = np.zeros(32 * 8, np.float32)
    d = float(ocean["level"] - y0 if depth is None else depth)
    f = abi.bind(load_library()[0], "st_", abi.OCEAN_FUNCS)
    n = f["ocean_waves"](C.byref(s), d, w.ctypes.data_as(abi.f32p))
    del keep
    return w[:n * 8].reshape(n, 8)


class FlipSim:
    """The FLIP water solver on a sparse MAC grid of 8^3 tiles (src/flip/sim.js:46)."""

    _prefix = "st_"

    def __init__(self, d, maxN, size=None, open=0, ratio=2.0, spray_cap=0, device=0, _funcs=None):
        self.f = _funcs if _funcs is not None else load_library()[1]
        desc = abi.FlipDesc()
        desc.size = C.sizeof(abi.FlipDesc)
        desc.d = float(d)
        desc.ratio = float(ratio or 2.0)
        sz = size or (3.0, 2.6, 3.0)
        desc.box[:] = [float(x) for x in sz]
        desc.open = int(open)
        desc.max_n = int(maxN)
        desc.spray_cap = int(spray_cap)
        desc.device = int(device)
        h = C.c_void_p()
        self._check(self.f["flip_create"](C.byref(desc), C.byref(h)), "create")
        self._h = h
        dims = abi.Dims()
        self.f["flip_get_dims"](self._h, C.byref(dims))
        self.d = float(d)
        self.ratio = max(1.4, min(4.0, float(ratio or 2.0)))
        self.h = float(dims.h)
        self.rest = self.ratio ** 3
        self.nx, self.ny, self.nz = dims.nx, dims.ny, dims.nz
        self.tx, self.ty, self.tz = dims.tx, dims.ty, dims.tz
        self.ntiles = self.tx * self.ty * self.tz
        self.ncell = self.nx * self.ny * self.nz
        self.b = dict(x0=dims.x0, y0=dims.y0, z0=dims.z0, x1=dims.x1, y1=dims.y1, z1=dims.z1)
        self.size = [self.nx * self.h, self.ny * self.h, self.nz * self.h]
        self.open = int(open)
        self.MAXN = int(maxN)
        self.cap = int(maxN)
        self.sprayCap = int(spray_cap)
        self.opt = {"noFoam": False, "noCull": False, "fastAir": False, "iters": 0}
        self.stats = None
        self.lastMs = 0.0     # track(): median device ms of the last 31 finished steps
        self.slowMs = 0.0     # the slowest step so far
        self.inflight = 0     # steps queued and not yet finished
        self._pend_p, self._pend_v = [], []
        self._n_host = 0

    def _check(self, st, what):
        if st not in (abi.ST_OK, abi.ST_NOT_READY):
            msg = ""
            if "last_error" in self.f:
                e = self.f["last_error"]()
                msg = e.decode() if e else ""
            raise StError("%s failed: %s %s" % (what, abi.STATUS_NAMES[st] if st < len(abi.STATUS_NAMES) else st, msg))
        return st

    @property
    def N(self):
        self.flushRun()
        s = abi.Stats()
        self._check(self.f["flip_stats"](self._h, C.byref(s)), "stats")
        return s.n

    def setCap(self, c):
        self.flushRun()
        self.cap = min(int(c), self.MAXN)
        self._check(self.f["flip_set_cap"](self._h, self.cap), "setCap")

    def clear(self):
        self._pend_p, self._pend_v = [], []
        self._check(self.f["flip_clear"](self._h), "clear")

    def add(self, x, y, z, vx, vy, vz):
        """FlipSim.add (src/gpu.js:390-402); buffered until flushRun."""
        self._pend_p.append((x, y, z))
        self._pend_v.append((vx, vy, vz))
        return True

    def add_many(self, pos3, vel3=None):
        """Many add() calls at once; returns how many were taken."""
        self.flushRun()
        p = np.ascontiguousarray(pos3, dtype=np.float32).reshape(-1, 3)
        v = np.zeros_like(p) if vel3 is None else np.ascontiguousarray(vel3, dtype=np.float32).reshape(-1, 3)
        got = C.c_uint32()
        self._check(self.f["flip_add"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), len(p), C.byref(got)), "add")
        return got.value

    def flushRun(self):
        if not self._pend_p:
            return
        p, v = self._pend_p, self._pend_v
        self._pend_p, self._pend_v = [], []
        self.add_many(np.array(p, np.float32), np.array(v, np.float32))

    def fillBox(self, x0, x1, y0, y1, z0, z1, rng=None):
        """FluidSim.fillBox (src/shared.js:285-291) with a seeded jitter source."""
        rng = rng or np.random.default_rng(0)
        d = self.d
        j = 0.01 * d / 0.12
        ys = np.arange(y0 + d / 2, y1, d)
        xs = np.arange(x0 + d / 2, x1, d)
        zs = np.arange(z0 + d / 2, z1, d)
        Y, X, Z = np.meshgrid(ys, xs, zs, indexing="ij")
        p = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        p = p + (rng.random(p.shape) - 0.5) * j
        return self.add_many(p)

    def fillSphere(self, cx, cy, cz, R, vx=0, vy=0, vz=0, rng=None):
        """FluidSim.fillSphere (src/shared.js:292-297) with a seeded jitter source."""
        rng = rng or np.random.default_rng(0)
        d = self.d
        j = 0.01 * d / 0.12
        r = np.arange(-R, R + 1e-12, d)
        Y, X, Z = np.meshgrid(r, r, r, indexing="ij")
        m = X ** 2 + Y ** 2 + Z ** 2 <= R * R
        p = np.stack([X[m] + cx, Y[m] + cy, Z[m] + cz], 1)
        p = p + (rng.random(p.shape) - 0.5) * j
        v = np.tile(np.array([vx, vy, vz], np.float32), (len(p), 1))
        return self.add_many(p, v)

    def step(self, dt, o):
        """FlipSim.step (src/flip/sim.js:179-241); returns the number of colliders used."""
        self.flushRun()
        s, keep = make_opts(o, self.opt)
        st = self.f["flip_step"](self._h, float(dt), C.byref(s))
        self._check(st, "step")
        del keep
        self.track()
        return min(len(o.get("cols") or []), 32)

    def track(self):
        """track (src/gpu.js:444-454): refresh lastMs (median device time of the last 31 finished steps), slowMs and
        inflight from the steps that have finished, without waiting for the rest."""
        if "flip_track" not in self.f:
            return
        n, last, slow = C.c_uint32(), C.c_float(), C.c_float()
        self._check(self.f["flip_track"](self._h, C.byref(n), C.byref(last), C.byref(slow)), "track")
        self.inflight, self.lastMs, self.slowMs = n.value, last.value, slow.value

    def stepTimed(self, dt, o):
        """FlipSim.stepTimed (src/flip/sim.js:312-331): device ms per stage."""
        self.flushRun()
        s, keep = make_opts(o, self.opt)
        t = abi.StageTimes()
        self._check(self.f["flip_step_timed"](self._h, float(dt), C.byref(s), C.byref(t)), "stepTimed")
        del keep
        return {n: getattr(t, n) for n in abi.STAGES}

    def read_frame(self, vs=1.0, out=None):
        """The particles as a cache frame (packFrameBuf, src/gpu.js:525-560), packed on the device: dict n, pos
        (n, 3) uint16, spd (n,) uint8 and fm (n,) uint8 or None when no point has white water. out: optional
        (pos, spd, fm) arrays with room for MAXN points (e.g. views of pinned host memory) to read into."""
        self.flushRun()
        cap = max(self.MAXN, 1)
        if out is None:
            pos, spd, fm = np.zeros((cap, 3), np.uint16), np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        else:
            pos, spd, fm = out
            cap = min(cap, len(spd), len(fm), pos.size // 3)
        n, foam = C.c_uint32(), C.c_int32()
        self._check(self.f["flip_read_frame"](self._h, float(vs), pos.ctypes.data_as(C.POINTER(C.c_uint16)), spd.ctypes.data_as(abi.u8p),
                                              fm.ctypes.data_as(abi.u8p), cap, C.byref(n), C.byref(foam)), "read_frame")
        m = n.value
        return dict(n=m, pos=pos[:m], spd=spd[:m], fm=fm[:m] if foam.value else None)

    def read_frame_async(self, vs=1.0, out=None):
        """Starts the same frame and returns at once (readbackInto's mapAsync, src/gpu.js:430-443): it is packed on the
        step stream and copied on a second stream while later steps run; frame_wait() gives it. out as in read_frame
        (pinned host memory lets the copy overlap the steps); the arrays are held until the wait."""
        self.flushRun()
        cap = max(self.MAXN, 1)
        if out is None:
            out = (np.zeros((cap, 3), np.uint16), np.zeros(cap, np.uint8), np.zeros(cap, np.uint8))
        pos, spd, fm = out
        cap = min(cap, len(spd), len(fm), pos.size // 3)
        self._frame_out = out
        self._check(self.f["flip_read_frame_async"](self._h, float(vs), pos.ctypes.data_as(C.POINTER(C.c_uint16)),
                                                    spd.ctypes.data_as(abi.u8p), fm.ctypes.data_as(abi.u8p), cap), "read_frame_async")

    def frame_wait(self):
        """The frame of the last read_frame_async once it has landed, as read_frame returns it (n = 0 when none is
        pending)."""
        n, foam = C.c_uint32(), C.c_int32()
        self._check(self.f["flip_frame_wait"](self._h, C.byref(n), C.byref(foam)), "frame_wait")
        out, self._frame_out = getattr(self, "_frame_out", None), None
        m = n.value
        if out is None:
            return dict(n=0, pos=np.zeros((0, 3), np.uint16), spd=np.zeros(0, np.uint8), fm=None)
        pos, spd, fm = out
        return dict(n=m, pos=pos[:m], spd=spd[:m], fm=fm[:m] if foam.value else None)

    def bake_diag(self, vcap=14.0):
        """bakeDiag (src/flip/bake.js:60-83) computed on the device, with the reference's keys."""
        d = abi.BakeDiag()
        self._check(self.f["flip_bake_diag"](self._h, float(vcap or 0.0), C.byref(d)), "bake_diag")
        return dict(alive=d.alive, gone=d.gone, nonFinite=d.non_finite, outsideBox=d.outside_box, atWaterSpeedLimit=d.at_speed_limit,
                    meanSpeed=d.mean_speed, maxSpeed=d.max_speed, meanFoam=d.mean_foam, foamyPoints=d.foamy, center=list(d.center),
                    bbox=list(d.bbox) if d.has_bbox else None, heightHist=list(d.height_hist))

    def save_full(self):
        """The full checkpoint (st_flip_save_full) as bytes."""
        self.flushRun()
        n = C.c_uint64()
        self._check(self.f["flip_save_full"](self._h, None, 0, C.byref(n)), "save_full")
        buf = C.create_string_buffer(n.value)
        self._check(self.f["flip_save_full"](self._h, buf, n.value, C.byref(n)), "save_full")
        return buf.raw

    def load_full(self, blob):
        """Restore a full checkpoint made by a simulator with the same geometry and capacity."""
        self._pend_p, self._pend_v = [], []
        self._check(self.f["flip_load_full"](self._h, blob, len(blob)), "load_full")

    def set_launch(self, tile_ctas_per_sm, light_ctas_per_sm, sor_ctas_per_sm):
        """CTAs per SM of the heavy per-tile kernels, the light ones and the pressure sweeps (st_flip_set_launch)."""
        self._check(self.f["flip_set_launch"](self._h, int(tile_ctas_per_sm), int(light_ctas_per_sm), int(sor_ctas_per_sm)),
                    "set_launch")

    def set_timing(self, on=True):
        """Record per-stage device times of every step without stalling (st_flip_set_timing)."""
        self._check(self.f["flip_set_timing"](self._h, 1 if on else 0), "set_timing")

    def read_timing(self):
        """Summed stage ms of the steps recorded since set_timing/read_timing, and how many steps that is."""
        t = abi.StageTimes()
        n = C.c_uint32()
        self._check(self.f["flip_read_timing"](self._h, C.byref(t), C.byref(n)), "read_timing")
        return {k: getattr(t, k) for k in abi.STAGES}, n.value

    def readStats(self):
        s = abi.Stats()
        self._check(self.f["flip_stats"](self._h, C.byref(s)), "stats")
        return self._set_stats(s)

    def _set_stats(self, s):
        self.stats = dict(sc=s.sc, ovf=s.ovf, fluid=s.fluid, vmax=s.vmax, n=s.n, live=s.live, spray_used=s.spray_used, steps=s.steps,
                          spray_overflow=s.spray_overflow, launches=s.launches)
        return self.stats

    def readStatsAsync(self):
        """readStats as the reference issues it (src/flip/sim.js:160-168): the counters' copy is queued behind the work
        so far and the call returns a ticket; statsWait(ticket) gives them once they have landed."""
        t = C.c_uint64()
        self._check(self.f["flip_stats_async"](self._h, C.byref(t)), "readStatsAsync")
        return t.value

    def statsWait(self, ticket):
        s = abi.Stats()
        self._check(self.f["flip_stats_wait"](self._h, C.c_uint64(ticket), C.byref(s)), "statsWait")
        return self._set_stats(s)

    def activeCells(self):
        return self.readStats()["fluid"]

    def readbackInto(self, dst=None, vel=None):
        """Particles in id order (src/flip/sim.js:439-455); returns (n, pos4[, vel4])."""
        self.flushRun()
        n = self.N
        if dst is None:
            dst = np.zeros((max(n, 1), 4), np.float32)
        pv = None if vel is None else vel.ctypes.data_as(abi.f32p)
        got = C.c_uint32()
        self._check(self.f["flip_read_particles"](self._h, dst.ctypes.data_as(abi.f32p), pv, dst.size // 4, C.byref(got)), "readback")
        return got.value

    def particles(self):
        n = self.N
        p = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 4), np.float32)
        got = C.c_uint32()
        self._check(self.f["flip_read_particles"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), n, C.byref(got)), "readback")
        return p, v

    def readSpray(self):
        """FlipSim.readSpray (src/flip/sim.js:423-437)."""
        if not self.sprayCap:
            return None
        p = np.zeros((self.sprayCap, 4), np.float32)
        v = np.zeros((self.sprayCap, 4), np.float32)
        n = C.c_uint32()
        self._check(self.f["flip_read_spray"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), self.sprayCap, C.byref(n)), "readSpray")
        return dict(n=n.value, p=p[: n.value], v=v[: n.value])

    def setSprayCap(self, n):
        """FlipSim.setSprayCap (src/flip/sim.js:326-334): room for n whitewater points (0 turns whitewater off)."""
        self.flushRun()
        self._check(self.f["flip_set_spray_cap"](self._h, int(n)), "setSprayCap")
        self.sprayCap = int(n)

    @property
    def recycle(self):
        """FlipSim.recycle: add() reuses slots in a ring once the cap is reached (default on)."""
        return getattr(self, "_recycle", True)

    @recycle.setter
    def recycle(self, on):
        self._check(self.f["flip_set_recycle"](self._h, 1 if on else 0), "recycle")
        self._recycle = bool(on)

    def prime(self, o=None):
        """FlipSim.prime (src/flip/sim.js:170-178) sizes the reference's block pool for the starting water. Every tile
        here has a fixed home in device memory, so there is no pool to size: nothing to do."""
        return None

    def memBytes(self):
        """FlipSim.memBytes (src/flip/sim.js:492-495): device memory this simulator holds."""
        b = C.c_uint64()
        self._check(self.f["flip_mem_bytes"](self._h, C.byref(b)), "memBytes")
        return b.value

    def readDeep(self):
        """FlipSim.readDeep (src/flip/sim.js:408-421): dict n, p ((n, 4) float32: x, y, z, 4096 + speed) of the deep
        water of the last step, or None when the deep look does not apply."""
        self.flushRun()
        out = np.zeros((200000, 4), np.float32)
        n = C.c_uint32()
        self._check(self.f["flip_read_deep_points"](self._h, out.ctypes.data_as(abi.f32p), len(out), C.byref(n)), "readDeep")
        return dict(n=n.value, p=out[:n.value]) if n.value else None

    def pump(self, vs=1.0):
        """FlipSim.pump + unpackLive (src/flip/sim.js:506-537): the live view packed on the device, read back and made
        into this.outFrame (n, pos, spd, fm, b, and sp / dp when present); gen counts the frames made."""
        words, L = self.pack_live(vs)
        u8, u16 = words.view(np.uint8), words.view(np.uint16)
        nW, nS, nD = L["n_water"], min(int(words[0]), L["n_spray"]), min(int(words[1]), L["n_deep"])
        fr = dict(n=nW, pos=u16[L["o_wp"] * 2: L["o_wp"] * 2 + nW * 3].reshape(nW, 3).copy(), spd=u8[L["o_ws"] * 4: L["o_ws"] * 4 + nW].copy(),
                  fm=u8[L["o_wf"] * 4: L["o_wf"] * 4 + nW].copy(), b=dict(self.b))
        if nS:
            fr["sp"] = dict(n=nS, pos=u16[L["o_sp"] * 2: L["o_sp"] * 2 + nS * 3].reshape(nS, 3).copy(), pk=words[L["o_sk"]: L["o_sk"] + nS].copy(), alive=nS)
        if nD:
            fr["dp"] = dict(n=nD, pos=u16[L["o_dp"] * 2: L["o_dp"] * 2 + nD * 3].reshape(nD, 3).copy(), spd=u8[L["o_ds"] * 4: L["o_ds"] * 4 + nD].copy())
        self.outFrame = fr
        self.gen = getattr(self, "gen", 0) + 1
        return fr

    def setDeepLook(self, on):
        """FlipSim.setDeepLook (src/flip/sim.js:406): show the narrow band's deep water as points."""
        self._check(self.f["flip_set_deep_look"](self._h, 1 if on else 0), "setDeepLook")

    def read_deep(self, vs=1.0):
        """readDeep + packDeep (src/flip/sim.js:408-421, src/gpu.js:512-524) on the device: the frame's deep-water part,
        dict n, pos (n, 3) uint16 and spd (n,) uint8, or None when the deep look does not apply."""
        self.flushRun()
        cap = 200000
        pos, spd = np.zeros((cap, 3), np.uint16), np.zeros(cap, np.uint8)
        n = C.c_uint32()
        self._check(self.f["flip_read_deep"](self._h, float(vs), pos.ctypes.data_as(C.POINTER(C.c_uint16)), spd.ctypes.data_as(abi.u8p), cap,
                                             C.byref(n)), "readDeep")
        m = n.value
        return dict(n=m, pos=pos[:m], spd=spd[:m]) if m else None

    def read_spray_frame(self, cap=200000, foam_life=3.0):
        """packSprayFrame (src/flip/bake.js:43-58) on the device: the frame's whitewater part, dict n, pos (n, 3) uint16,
        pk (n,) uint32 and alive, or None without a whitewater pool."""
        if not self.sprayCap:
            return None
        self.flushRun()
        room = self.sprayCap
        pos, pk = np.zeros((room, 3), np.uint16), np.zeros(room, np.uint32)
        n, alive = C.c_uint32(), C.c_uint32()
        self._check(self.f["flip_read_spray_frame"](self._h, int(cap), float(foam_life), pos.ctypes.data_as(C.POINTER(C.c_uint16)),
                                                    pk.ctypes.data_as(abi.u32p), room, C.byref(n), C.byref(alive)), "readSprayFrame")
        m = n.value
        return dict(n=m, pos=pos[:m], pk=pk[:m], alive=alive.value)

    def pack_live(self, vs=1.0):
        """FlipSim.dispPack (src/flip/sim.js:381-404) on the device: (words, layout) of the packed live view."""
        self.flushRun()
        L = abi.LiveLayout()
        L.size = C.sizeof(abi.LiveLayout)
        self._check(self.f["flip_pack_live"](self._h, float(vs), None, 0, C.byref(L)), "packLive")
        words = np.zeros(max(L.words, 1), np.uint32)
        self._check(self.f["flip_pack_live"](self._h, float(vs), words.ctypes.data_as(abi.u32p), len(words), C.byref(L)), "packLive")
        return words[:L.words], {k: getattr(L, k) for k, _ in abi.LiveLayout._fields_ if k != "size"}

    def read_air(self):
        """The air field: (nz, ny, nx, 3) float32 air velocity at the air-cell centres, or None without a whitewater pool."""
        dims = (C.c_uint32 * 3)()
        self._check(self.f["flip_read_air"](self._h, None, 0, dims), "readAir")
        nx, ny, nz = dims[0], dims[1], dims[2]
        if not nx:
            return None
        a = np.zeros((nz * ny * nx, 4), np.float32)
        self._check(self.f["flip_read_air"](self._h, a.ctypes.data_as(abi.f32p), nx * ny * nz, dims), "readAir")
        return a[:, :3].reshape(nz, ny, nx, 3)

    def read_drips(self):
        """The drip samples: (n, 8) float32 rows of local position, collider number, local normal, wetness."""
        n = C.c_uint32()
        self._check(self.f["flip_read_drips"](self._h, None, 0, C.byref(n)), "readDrips")
        a = np.zeros((n.value, 8), np.float32)
        if n.value:
            self._check(self.f["flip_read_drips"](self._h, a.ctypes.data_as(abi.f32p), n.value, C.byref(n)), "readDrips")
        return a

    def grid(self):
        """Every cell of the tile box: tile_on, cnt, ctype, pres, rhs, vn, vo, velg (dense numpy arrays)."""
        NX, NY, NZ = self.tx * 8, self.ty * 8, self.tz * 8
        nc = NX * NY * NZ
        out = dict(tile_on=np.zeros(self.ntiles, np.uint8), cnt=np.zeros(nc, np.int32), ctype=np.zeros(nc, np.uint32),
                   pres=np.zeros(nc, np.float32), rhs=np.zeros(nc, np.float32), vn=np.zeros(nc * 3, np.float32),
                   vo=np.zeros(nc * 3, np.float32), velg=np.zeros(nc * 3, np.float32))
        g = abi.Grid()
        g.tile_on = out["tile_on"].ctypes.data_as(abi.u8p)
        g.cnt = out["cnt"].ctypes.data_as(abi.i32p)
        g.ctype = out["ctype"].ctypes.data_as(abi.u32p)
        for k in ("pres", "rhs", "vn", "vo", "velg"):
            setattr(g, k, out[k].ctypes.data_as(abi.f32p))
        self._check(self.f["flip_read_grid"](self._h, C.byref(g)), "read_grid")
        shp = (NZ, NY, NX)
        for k in ("cnt", "ctype", "pres", "rhs"):
            out[k] = out[k].reshape(shp)
        for k in ("vn", "vo", "velg"):
            out[k] = out[k].reshape(shp + (3,))
        return out

    def save_state(self):
        """(pos4, vel4, pid) in storage order."""
        n = self.N
        p = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 4), np.float32)
        i = np.zeros(n, np.uint32)
        got = C.c_uint32()
        self._check(self.f["flip_save_state"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p),
                                              i.ctypes.data_as(abi.u32p), n, C.byref(got)), "save_state")
        return p, v, i

    def load_state(self, pos4, vel4, pid, t=0.0, seed=0):
        p = np.ascontiguousarray(pos4, np.float32).reshape(-1, 4)
        v = np.ascontiguousarray(vel4, np.float32).reshape(-1, 4)
        i = np.ascontiguousarray(pid, np.uint32).reshape(-1)
        self._check(self.f["flip_load_state"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p),
                                              i.ctypes.data_as(abi.u32p), len(p), float(t), int(seed)), "load_state")

    def nb_fills(self, boxes=(), spheres=(), mode=1):
        """Starting water of the narrow band (sim.nbFills written by nbSeed, src/shared.js:849-851)."""
        b = np.ascontiguousarray(np.array(boxes, np.float32).reshape(-1, 6))
        s = np.ascontiguousarray(np.array(spheres, np.float32).reshape(-1, 4))
        self._check(self.f["flip_nb_fills"](self._h, b.ctypes.data_as(abi.f32p), len(b), s.ctypes.data_as(abi.f32p), len(s), int(mode)), "nb_fills")

    def nb_fill_vols(self, vols=(), mode=1):
        """Water meshes of the narrow band's start (sim.nbFillVols written by nbSeed, src/shared.js:829-831, 849-850):
        collider-shaped dicts (sdf, x, y, z, R) whose negative distance is water; the next restart step reads them."""
        pack = _ColliderPack(list(vols))
        self._check(self.f["flip_nb_fill_vols"](self._h, C.cast(pack.arr, C.POINTER(abi.Collider)), pack.n, int(mode)), "nb_fill_vols")

    def stream(self):
        return self.f["flip_stream"](self._h)

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["flip_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
