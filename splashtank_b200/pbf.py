"""PbfSim: the app's WebGPU position-based fluid engine (GpuSim, src/gpu.js:357-476) over st_pbf_* of the C ABI.

The surface follows the JavaScript class: ``step(dt, o)`` with the reference's options {g, iters, visc, cols} (cols are
the same collider dicts as FlipSim's: a signed distance grid ``sdf`` and a pose), ``add``, ``fillBox``,
``fillSphere``, ``setCap``, ``clear``, ``recycle``, ``readbackInto``, ``N``, ``MAXN``, ``d``, ``h``, ``b``.
Compute runs in libsplashtank_cuda.so; there is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import abi
from .flip import _ColliderPack, load_library, status_error

_PBF = None


def pbf_funcs():
    global _PBF
    if _PBF is None:
        _PBF = abi.bind(load_library()[0], "st_", abi.PBF_FUNCS)
    return _PBF


def pbf_opts(o):
    """GpuSim.step's options (src/gpu.js:409-416) as an st_pbf_opts; returns (opts, keepalive)."""
    cols = _ColliderPack(o.get("cols") or [])
    op = abi.PbfOpts()
    op.size = C.sizeof(abi.PbfOpts)
    op.g = float(o.get("g", 9.81))
    op.visc = float(o.get("visc", 0.0))
    op.iters = int(o.get("iters", 3))
    op.ncols = cols.n
    op.cols = C.cast(cols.arr, C.POINTER(abi.Collider))
    return op, cols


class PbfSim:
    def __init__(self, d, maxN, size=None, open=0, device=0, eps_k=0.0, wall_k=0.0, _funcs=None):
        self.f = _funcs if _funcs is not None else pbf_funcs()
        desc = abi.PbfDesc()
        desc.size = C.sizeof(abi.PbfDesc)
        desc.d = float(d)
        sz = size or (3.0, 2.6, 3.0)
        desc.box[:] = [float(x) for x in sz]
        desc.open = int(open)
        desc.max_n = int(maxN)
        desc.device = int(device)
        desc.eps_k = float(eps_k)
        desc.wall_k = float(wall_k)
        h = C.c_void_p()
        self._check(self.f["pbf_create"](C.byref(desc), C.byref(h)), "create")
        self._h = h
        self.d = float(d)
        self.h = 2.2 * self.d
        self.MAXN = int(maxN)
        self.cap = int(maxN)
        self.b = dict(x0=-sz[0] / 2, x1=sz[0] / 2, y0=0.0, y1=sz[1], z0=-sz[2] / 2, z1=sz[2] / 2)
        self.n = 0
        self._recycle = True

    def _check(self, st, what):
        if st not in (abi.ST_OK, abi.ST_NOT_READY):
            raise status_error("pbf " + what, st)

    @property
    def N(self):
        return self.n

    @property
    def recycle(self):
        return self._recycle

    @recycle.setter
    def recycle(self, on):
        self._check(self.f["pbf_set_recycle"](self._h, 1 if on else 0), "set_recycle")
        self._recycle = bool(on)

    def setCap(self, c):
        self._check(self.f["pbf_set_cap"](self._h, int(c)), "set_cap")
        self.cap = min(int(c), self.MAXN)
        self.n = min(self.n, self.cap)

    def clear(self):
        self._check(self.f["pbf_clear"](self._h), "clear")
        self.n = 0

    def add_many(self, pos3, vel3=None):
        p = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
        v = None if vel3 is None else np.ascontiguousarray(vel3, np.float32).reshape(-1, 3)
        got = C.c_uint32()
        self._check(self.f["pbf_add"](self._h, p.ctypes.data_as(abi.f32p), None if v is None else v.ctypes.data_as(abi.f32p), len(p),
                                      C.byref(got)), "add")
        self.n = min(self.cap, self.n + got.value)
        return got.value

    def add(self, x, y, z, vx=0.0, vy=0.0, vz=0.0):
        return self.add_many([[x, y, z]], [[vx, vy, vz]]) == 1

    def fillBox(self, x0, x1, y0, y1, z0, z1, rng=None):
        """FluidSim.fillBox (src/shared.js:285-291): a lattice at spacing d with a jitter of 0.01 d / 0.12, seeded."""
        rng = rng or np.random.default_rng(0)
        d = self.d
        j = 0.01 * d / 0.12
        ys, xs, zs = np.arange(y0 + d / 2, y1, d), np.arange(x0 + d / 2, x1, d), np.arange(z0 + d / 2, z1, d)
        Y, X, Z = np.meshgrid(ys, xs, zs, indexing="ij")
        p = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        return self.add_many(p + (rng.random(p.shape) - 0.5) * j)

    def fillSphere(self, cx, cy, cz, R, vx=0.0, vy=0.0, vz=0.0, rng=None):
        """FluidSim.fillSphere (src/shared.js:292-297), seeded jitter."""
        rng = rng or np.random.default_rng(0)
        d = self.d
        j = 0.01 * d / 0.12
        a = np.arange(-R, R + 1e-9, d)
        Y, X, Z = np.meshgrid(a, a, a, indexing="ij")
        m = X * X + Y * Y + Z * Z <= R * R
        p = np.stack([cx + X[m], cy + Y[m], cz + Z[m]], 1)
        p = p + (rng.random(p.shape) - 0.5) * j
        return self.add_many(p, np.tile(np.array([[vx, vy, vz]], np.float32), (len(p), 1)))

    def step(self, dt, o):
        """GpuSim.step (src/gpu.js:409-428)."""
        op, keep = pbf_opts(o)
        self._check(self.f["pbf_step"](self._h, float(dt), C.byref(op)), "step")
        del keep

    def particles(self):
        """(positions xyz + speed, velocities) of the N slots in index order."""
        p = np.zeros((max(self.n, 1), 4), np.float32)
        v = np.zeros((max(self.n, 1), 4), np.float32)
        got = C.c_uint32()
        self._check(self.f["pbf_read"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), self.n, C.byref(got)), "read")
        return p[: self.n], v[: self.n]

    def readbackInto(self, dst):
        p, _ = self.particles()
        dst[: len(p)] = p
        return len(p)

    def stream(self):
        return self.f["pbf_stream"](self._h)

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["pbf_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
