"""Python handle on the CPU oracle (oracle/flip_oracle.cpp), for tests, smoke() and bench.py's CPU baseline only.

OracleFlipSim has the same methods as splashtank_b200.flip.FlipSim because the oracle library exports the same
C entry points under the prefix ``oracle_``.  The oracle is the checker, never the thing measured as the product.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from splashtank_b200 import abi
from splashtank_b200.flip import FlipSim

HERE = os.path.dirname(os.path.abspath(__file__))
_FUNCS = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle_flip.so"), os.path.join(HERE, "liboracle_pbf.so"),
                    os.path.join(HERE, "liboracle_poisson.so"), os.path.join(HERE, "liboracle_sdf.so")], check=True)


def funcs():
    global _FUNCS
    if _FUNCS is None:
        path = os.path.join(HERE, "liboracle_flip.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        f = abi.bind(lib, "oracle_", abi.FLIP_FUNCS)
        f["set_threads"] = lib.oracle_flip_set_threads
        f["set_threads"].argtypes = [C.c_void_p, C.c_int]
        f["set_threads"].restype = None
        f["spray_overflow"] = lib.oracle_flip_spray_overflow
        f["spray_overflow"].argtypes = [C.c_void_p]
        f["spray_overflow"].restype = C.c_uint32
        f["deep_points"] = lib.oracle_flip_deep_points
        f["deep_points"].argtypes = [C.c_void_p, abi.f32p, C.c_uint32, abi.u32p]
        f["deep_points"].restype = C.c_int
        _FUNCS = f
    return _FUNCS


class OracleFlipSim(FlipSim):
    def __init__(self, *a, threads=1, **k):
        super().__init__(*a, _funcs=funcs(), **k)
        self.set_threads(threads)

    def set_threads(self, n):
        self.f["set_threads"](self._h, int(n))

    def stepTimed(self, dt, o):
        raise NotImplementedError("the oracle has no stage timer")

    def deep_points(self):
        """One deep pass (deepClear + deepPick + deepFin): (n, 4) float32 points x, y, z, 4096 + speed, or None when the
        deep look does not apply."""
        n = C.c_uint32()
        out = np.zeros((200000, 4), np.float32)   # a pass writes at most 200,000 points
        self.f["deep_points"](self._h, out.ctypes.data_as(abi.f32p), len(out), C.byref(n))
        return out[:n.value].copy() if n.value else None


_PBF = None
_BAKER = None


def pbf_funcs():
    """oracle_pbf_*: the GpuSim restatement, bound with st_pbf_*'s signatures."""
    global _PBF
    if _PBF is None:
        path = os.path.join(HERE, "liboracle_pbf.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        f = abi.bind(lib, "oracle_", abi.PBF_FUNCS)
        f["set_threads"] = lib.oracle_pbf_set_threads
        f["set_threads"].argtypes = [C.c_void_p, C.c_int]
        f["set_threads"].restype = None
        _PBF = f
    return _PBF


from splashtank_b200.pbf import PbfSim  # noqa: E402


class OraclePbfSim(PbfSim):
    """The CPU restatement of GpuSim (oracle/pbf_oracle.cpp) behind PbfSim's methods."""

    def __init__(self, *a, threads=1, **k):
        super().__init__(*a, _funcs=pbf_funcs(), **k)
        self.f["set_threads"](self._h, int(threads))


class BakerDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("d", C.c_double), ("box", C.c_double * 3), ("max_n", C.c_uint32)]


class BakerCol(C.Structure):
    _fields_ = [("kind", C.c_int32)] + [(n, C.c_float) for n in ("x", "y", "z", "r", "hx", "hy", "hz", "yaw")]


class BakerOpts(C.Structure):
    _fields_ = [("size", C.c_uint32), ("g", C.c_float), ("visc", C.c_float), ("iters", C.c_int32), ("ncols", C.c_uint32),
                ("cols", C.POINTER(BakerCol))]


def baker_funcs():
    global _BAKER
    if _BAKER is None:
        path = os.path.join(HERE, "liboracle_baker.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        sig = {"create": (C.c_int, [C.POINTER(BakerDesc), C.POINTER(C.c_void_p)]), "destroy": (None, [C.c_void_p]),
               "set_threads": (None, [C.c_void_p, C.c_int]), "add": (C.c_int, [C.c_void_p, abi.f32p, abi.f32p, C.c_uint32, abi.u32p]),
               "fill_box": (C.c_uint32, [C.c_void_p] + [C.c_float] * 6), "step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(BakerOpts)]),
               "read": (C.c_int, [C.c_void_p, abi.f32p, abi.f32p, C.c_uint32, abi.u32p])}
        f = {}
        for k, (res, args) in sig.items():
            fn = getattr(lib, "oracle_baker_" + k)
            fn.restype, fn.argtypes = res, args
            f[k] = fn
        _BAKER = f
    return _BAKER


class OracleBakerSim:
    """The CPU restatement of native/splash.cpp's Sim (oracle/baker_oracle.cpp): analytic sphere and yawed box colliders
    {"kind": "sphere", x, y, z, r} / {"kind": "box", x, y, z, hx, hy, hz, yaw}, a 48-neighbour cap, closed walls."""

    def __init__(self, d, maxN, size=None, threads=1):
        self.f = baker_funcs()
        desc = BakerDesc()
        desc.size = C.sizeof(BakerDesc)
        desc.d = float(d)
        desc.box[:] = [float(x) for x in (size or (3.0, 2.6, 3.0))]
        desc.max_n = int(maxN)
        h = C.c_void_p()
        if self.f["create"](C.byref(desc), C.byref(h)) != abi.ST_OK:
            raise RuntimeError("baker oracle create failed")
        self._h = h
        self.f["set_threads"](self._h, int(threads))
        self.n = 0

    def fill_box_baker(self, x0, x1, y0, y1, z0, z1):
        """The baker's own fillBox (native/splash.cpp:85-89): lattice plus jitter from mt19937 seeded 12345."""
        n = self.f["fill_box"](self._h, x0, x1, y0, y1, z0, z1)
        self.n += n
        return n

    def add_many(self, pos3, vel3=None):
        p = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
        v = None if vel3 is None else np.ascontiguousarray(vel3, np.float32).reshape(-1, 3)
        got = C.c_uint32()
        self.f["add"](self._h, p.ctypes.data_as(abi.f32p), None if v is None else v.ctypes.data_as(abi.f32p), len(p), C.byref(got))
        self.n += got.value
        return got.value

    def step(self, dt, o):
        cols = o.get("cols") or []
        arr = (BakerCol * max(len(cols), 1))()
        for k, c in enumerate(cols):
            arr[k].kind = 1 if c.get("kind") == "box" else 0
            for f in ("x", "y", "z", "r", "hx", "hy", "hz", "yaw"):
                setattr(arr[k], f, float(c.get(f, 0.0)))
        op = BakerOpts()
        op.size = C.sizeof(BakerOpts)
        op.g, op.visc, op.iters, op.ncols = float(o.get("g", 9.8)), float(o.get("visc", 0.0)), int(o.get("iters", 3)), len(cols)
        op.cols = C.cast(arr, C.POINTER(BakerCol))
        self.f["step"](self._h, float(dt), C.byref(op))

    def particles(self):
        p = np.zeros((max(self.n, 1), 4), np.float32)
        v = np.zeros((max(self.n, 1), 4), np.float32)
        got = C.c_uint32()
        self.f["read"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p), self.n, C.byref(got))
        return p[:got.value], v[:got.value]

    def __del__(self):
        try:
            self.f["destroy"](self._h)
        except Exception:
            pass


class OraclePoisson:
    """FP32 SOR sweeps, FP64 residual norms (the kernels' summation order) and the all-FP64 CG reference solve."""

    def __init__(self, n, open=0, threads=8):
        lib = C.CDLL(os.path.join(HERE, "liboracle_poisson.so")) if os.path.exists(os.path.join(HERE, "liboracle_poisson.so")) else None
        if lib is None:
            build()
            lib = C.CDLL(os.path.join(HERE, "liboracle_poisson.so"))
        dp = C.POINTER(C.c_double)
        lib.oracle_poisson_create.restype = C.c_void_p
        lib.oracle_poisson_create.argtypes = [C.c_uint32] * 4 + [C.c_int]
        lib.oracle_poisson_destroy.argtypes = [C.c_void_p]
        lib.oracle_poisson_set.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), dp]
        lib.oracle_poisson_sweeps32.argtypes = [C.c_void_p, C.c_float, C.c_int, dp]
        lib.oracle_poisson_rel_residual.restype = C.c_double
        lib.oracle_poisson_rel_residual.argtypes = [C.c_void_p, dp, dp, dp]
        lib.oracle_poisson_cg.restype = C.c_int
        lib.oracle_poisson_cg.argtypes = [C.c_void_p, C.c_double, C.c_int, dp]
        self.lib = lib
        self.n = tuple(int(x) for x in n)
        self.h = lib.oracle_poisson_create(self.n[0], self.n[1], self.n[2], int(open), int(threads))

    def set(self, cell_type, rhs):
        self._t = np.ascontiguousarray(cell_type, np.uint8)
        self._b = np.ascontiguousarray(rhs, np.float64)
        self.lib.oracle_poisson_set(self.h, self._t.ctypes.data_as(C.POINTER(C.c_uint8)), self._b.ctypes.data_as(C.POINTER(C.c_double)))

    def sweeps32(self, omega, iters):
        out = np.zeros(self.n[::-1], np.float64)
        self.lib.oracle_poisson_sweeps32(self.h, float(omega), int(iters), out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def rel_residual(self, x):
        x = np.ascontiguousarray(x, np.float64)
        return self.lib.oracle_poisson_rel_residual(self.h, x.ctypes.data_as(C.POINTER(C.c_double)), None, None)

    def cg(self, tol=1e-12, maxit=100000):
        out = np.zeros(self.n[::-1], np.float64)
        it = self.lib.oracle_poisson_cg(self.h, float(tol), int(maxit), out.ctypes.data_as(C.POINTER(C.c_double)))
        return out, it

    def __del__(self):
        try:
            self.lib.oracle_poisson_destroy(self.h)
        except Exception:
            pass


_SDF = None


def build_sdf(v, faces, cell=0.025, margin=0.16):
    """The oracle's buildSDF (oracle/sdf_oracle.cpp), through the same wrapper as the device builder."""
    global _SDF
    if _SDF is None:
        path = os.path.join(HERE, "liboracle_sdf.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        _SDF = lib.oracle_build_sdf
        _SDF.argtypes = [C.POINTER(abi.Mesh), C.POINTER(abi.SdfBuild)]
        _SDF.restype = C.c_int
    from splashtank_b200.sdf import build_sdf as wrap
    return wrap(v, faces, cell, margin, fn=_SDF)
