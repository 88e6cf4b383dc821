"""The pressure projection's linear solve on its own (st_poisson_*): FP32 red-black SOR, FP32 SOR inside FP64 iterative
refinement, and FP64 SOR, for the precision study. Compute runs in libsplashtank_cuda.so."""
import ctypes as C

import numpy as np

from . import abi
from .flip import load_library, status_error

SOR32, REFINE, SOR64 = 0, 1, 2
_F = None


def funcs():
    global _F
    if _F is None:
        _F = abi.bind(load_library()[0], "st_", abi.POISSON_FUNCS)
    return _F


class PoissonSolver:
    def __init__(self, n, open=0, device=0):
        self.f = funcs()
        d = abi.PoissonDesc()
        d.size = C.sizeof(abi.PoissonDesc)
        d.n[:] = [int(x) for x in n]
        d.open = int(open)
        d.device = int(device)
        h = C.c_void_p()
        self._check(self.f["poisson_create"](C.byref(d), C.byref(h)), "create")
        self._h = h
        self.n = tuple(int(x) for x in n)

    def _check(self, st, what):
        if st != abi.ST_OK:
            raise status_error("poisson " + what, st)

    def set(self, cell_type, rhs):
        """cell_type: uint8 (nz, ny, nx) 0 air / 1 fluid / 2 solid; rhs: float64 same shape."""
        t = np.ascontiguousarray(cell_type, np.uint8)
        b = np.ascontiguousarray(rhs, np.float64)
        self._check(self.f["poisson_set"](self._h, t.ctypes.data_as(abi.u8p), b.ctypes.data_as(C.POINTER(C.c_double))), "set")
        n = t.shape
        occ = (t == 1).reshape(n[0] // 8, 8, n[1] // 8, 8, n[2] // 8, 8).any(axis=(1, 3, 5)) if all(x % 8 == 0 for x in n) else None
        self.n_tiles = int(occ.sum()) if occ is not None else None
        self.n_fluid = int((t == 1).sum())

    def solve(self, mode, tol=1e-6, omega=1.9, max_sweeps=100000, inner_sweeps=50, check_every=10):
        o = abi.PoissonOpts()
        o.size = C.sizeof(abi.PoissonOpts)
        o.mode, o.tol, o.omega, o.max_sweeps, o.inner_sweeps, o.check_every = int(mode), float(tol), float(omega), int(max_sweeps), int(inner_sweeps), int(check_every)
        r = abi.PoissonResult()
        self._check(self.f["poisson_solve"](self._h, C.byref(o), C.byref(r)), "solve")
        return dict(rel_residual=r.rel_residual, sweeps=r.sweeps, refinements=r.refinements, converged=bool(r.converged), ms=r.ms)

    def sweeps32(self, omega, iters):
        """iters FP32 SOR iterations from zero; returns their device time in ms."""
        ms = C.c_float(0.0)
        self._check(self.f["poisson_sweeps32"](self._h, float(omega), int(iters), C.byref(ms)), "sweeps32")
        return ms.value

    def stats(self):
        """(active tiles, fluid cells) of the current system."""
        return self.n_tiles, self.n_fluid

    def read(self):
        out = np.zeros(self.n[::-1], np.float64)
        self._check(self.f["poisson_read"](self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "read")
        return out

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["poisson_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
