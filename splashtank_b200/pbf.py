"""PbfSim: the reference's position-based fluid solver (GpuSim, src/gpu.js:357-476; FluidSim, src/shared.js:220-501;
native/splash.cpp Sim) over st_pbf_* of the C ABI.

step(dt, o) takes the reference's options {g, iters, visc, cols}; colliders are the native baker's analytic shapes:
{"kind": "sphere", x, y, z, r} or {"kind": "box", x, y, z, hx, hy, hz, yaw}. Compute runs in libsplashtank_cuda.so.
"""
import ctypes as C

import numpy as np

from . import abi
from .flip import load_library, status_error

_PBF = None


def pbf_funcs():
    global _PBF
    if _PBF is None:
        lib = load_library()[0]
        _PBF = abi.bind(lib, "st_", abi.PBF_FUNCS)
    return _PBF


def col_array(cols):
    arr = (abi.PbfCol * max(len(cols), 1))()
    for k, c in enumerate(cols):
        r = arr[k]
        r.kind = 1 if c.get("kind") == "box" else 0
        for f in ("x", "y", "z", "r", "hx", "hy", "hz", "yaw"):
            setattr(r, f, float(c.get(f, 0.0)))
    return arr


class PbfSim:
    def __init__(self, d, maxN, size=None, open=0, device=0, eps_k=0.0, wall_k=0.0, _funcs=None):
        self.f = _funcs if _funcs is not None else pbf_funcs()
        desc = abi.PbfDesc()
        desc.size = C.sizeof(abi.PbfDesc)
        desc.d = float(d)
        desc.box[:] = [float(x) for x in (size or (3.0, 2.6, 3.0))]
        desc.open = int(open)
        desc.max_n = int(maxN)
        desc.device = int(device)
        desc.eps_k = float(eps_k)
        desc.wall_k = float(wall_k)
        h = C.c_void_p()
        st = self.f["pbf_create"](C.byref(desc), C.byref(h))
        if st != abi.ST_OK:
            raise status_error("pbf create", st)
        self._h = h
        self.d = float(d)
        self.h = 2.2 * self.d
        self.MAXN = int(maxN)
        sz = size or (3.0, 2.6, 3.0)
        self.b = dict(x0=-sz[0] / 2, x1=sz[0] / 2, y0=0.0, y1=sz[1], z0=-sz[2] / 2, z1=sz[2] / 2)
        self.n = 0

    @property
    def N(self):
        return self.n

    def add_many(self, pos3, vel3=None):
        p = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
        v = None if vel3 is None else np.ascontiguousarray(vel3, np.float32).reshape(-1, 3)
        got = C.c_uint32()
        st = self.f["pbf_add"](self._h, p.ctypes.data_as(abi.f32p), None if v is None else v.ctypes.data_as(abi.f32p), len(p), C.byref(got))
        if st != abi.ST_OK:
            raise status_error("pbf add", st)
        self.n += got.value
        return got.value

    def add(self, x, y, z, vx=0.0, vy=0.0, vz=0.0):
        return self.add_many([[x, y, z]], [[vx, vy, vz]]) == 1

    def fillBox(self, x0, x1, y0, y1, z0, z1, rng=None):
        """Lattice fill with a small seeded jitter (FluidSim.fillBox, src/shared.js:285-291)."""
        rng = rng or np.random.default_rng(0)
        d = self.d
        j = 0.01 * d / 0.12
        ys, xs, zs = np.arange(y0 + d / 2, y1, d), np.arange(x0 + d / 2, x1, d), np.arange(z0 + d / 2, z1, d)
        Y, X, Z = np.meshgrid(ys, xs, zs, indexing="ij")
        p = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        return self.add_many(p + (rng.random(p.shape) - 0.5) * j)

    def step(self, dt, o):
        """GpuSim.step / Sim::step (src/gpu.js:409-428, native/splash.cpp:212-247)."""
        cols = o.get("cols") or []
        arr = col_array(cols)
        op = abi.PbfOpts()
        op.size = C.sizeof(abi.PbfOpts)
        op.g = float(o.get("g", 9.8))
        op.visc = float(o.get("visc", 0.0))
        op.iters = int(o.get("iters", 3))
        op.ncols = len(cols)
        op.cols = C.cast(arr, C.POINTER(abi.PbfCol))
        st = self.f["pbf_step"](self._h, float(dt), C.byref(op))
        if st not in (abi.ST_OK, abi.ST_NOT_READY):
            raise status_error("pbf step", st)

    def particles(self):
        p = np.zeros((max(self.n, 1), 4), np.float32)
        v = np.zeros((max(self.n, 1), 4), np.float32)
        got = C.c_uint32()
        st = self.f["pbf_read"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), self.n, C.byref(got))
        if st != abi.ST_OK:
            raise status_error("pbf read", st)
        return p[: got.value], v[: got.value]

    def readbackInto(self, dst):
        p, _ = self.particles()
        dst[: len(p)] = p
        return len(p)

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["pbf_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
