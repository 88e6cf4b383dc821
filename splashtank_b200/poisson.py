"""The pressure projection's linear solve on its own (st_poisson_*): FP32 red-black SOR, FP32 SOR inside FP64 iterative
refinement, and FP64 SOR, for the precision study. Compute runs in libsplashtank_cuda.so."""
import ctypes as C

import numpy as np

from . import abi
from .flip import load_library, status_error

SOR32, REFINE, SOR64 = 0, 1, 2
_F = None
_NA = None


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

    def solve(self, mode, tol=1e-6, omega=1.9, max_sweeps=100000, inner_sweeps=50, check_every=10, predict=False):
        """predict: size each block of iterations between residual checks from the last block's reduction (the same
        rule for every mode), instead of fixed blocks."""
        o = abi.PoissonOpts()
        o.size = C.sizeof(abi.PoissonOpts)
        o.mode, o.tol, o.omega, o.max_sweeps, o.inner_sweeps, o.check_every = int(mode), float(tol), float(omega), int(max_sweeps), int(inner_sweeps), int(check_every)
        o.schedule = 1 if predict else 0
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


# ---------------------------------------------------------------- the system in the tile-major layout, on the host
def _tile_index(n):
    """Tile-major index of every cell of a dense (nz, ny, nx) box: t * 512 + lx + 8 (ly + 8 lz)."""
    nx, ny, nz = n
    tx, ty = (nx + 7) // 8, (ny + 7) // 8
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    t = (i >> 3) + tx * ((j >> 3) + ty * (k >> 3))
    return (t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7))).astype(np.int64)


def n_cells(n):
    return ((n[0] + 7) // 8) * ((n[1] + 7) // 8) * ((n[2] + 7) // 8) * 512


def to_tile_major(dense):
    """A dense (nz, ny, nx) field in the tile-major layout (zeros in the cells past the box)."""
    n = dense.shape[::-1]
    out = np.zeros(n_cells(n), dense.dtype)
    out[_tile_index(n).ravel()] = dense.ravel()
    return out


def tile_system(cell_type, rhs, open=0):
    """(tiles, info, b) of st_poisson_system built on the host, as st_poisson_set builds them: tiles holding fluid
    ascending; info = 0x8000 | non-solid neighbours << 8 | fluid-neighbour bits (-x, +x, -y, +y, -z, +z), the box's
    outside solid unless its face is open (ST_OPEN_* bits); b = rhs on fluid cells."""
    t = np.ascontiguousarray(cell_type, np.uint8)
    nz, ny, nx = t.shape
    fluid = t == 1
    pad = np.full((nz + 2, ny + 2, nx + 2), 2, np.uint8)
    pad[1:-1, 1:-1, 1:-1] = t
    for bit, sl in ((1, np.s_[1:-1, 1:-1, 0]), (2, np.s_[1:-1, 1:-1, -1]), (4, np.s_[1:-1, 0, 1:-1]), (8, np.s_[1:-1, -1, 1:-1]),
                    (16, np.s_[0, 1:-1, 1:-1]), (32, np.s_[-1, 1:-1, 1:-1])):
        if open & bit:
            pad[sl] = 0
    nbs = [pad[1:-1, 1:-1, :-2], pad[1:-1, 1:-1, 2:], pad[1:-1, :-2, 1:-1], pad[1:-1, 2:, 1:-1], pad[:-2, 1:-1, 1:-1], pad[2:, 1:-1, 1:-1]]
    mask = np.zeros(t.shape, np.uint16)
    nns = np.zeros(t.shape, np.uint16)
    for a, q in enumerate(nbs):
        mask |= (q == 1).astype(np.uint16) << a
        nns += (q != 2).astype(np.uint16)
    info = np.where(fluid, 0x8000 | (nns << 8) | mask, 0).astype(np.uint16)
    b = np.where(fluid, np.asarray(rhs, np.float64), 0.0)
    idx = _tile_index((nx, ny, nz))
    tiles = np.unique(idx[fluid] >> 9).astype(np.uint32)
    return tiles, to_tile_major(info), to_tile_major(b)


def residual_noalloc(n, tiles, info, b, x, stream=0):
    """st_poisson_residual_noalloc on device arrays (anything with data_ptr(), e.g. torch CUDA tensors: tiles uint32
    (int32 storage), info uint16 (int16 storage), b and x float64 in the tile-major layout). Returns (rel, r2, b2)."""
    global _NA
    if _NA is None:
        _NA = abi.bind(load_library()[0], "st_", abi.NOALLOC_FUNCS)
    s = abi.PoissonSystem()
    s.size = C.sizeof(abi.PoissonSystem)
    s.n[:] = [int(v) for v in n]
    s.n_tiles = int(tiles.numel())
    s.tiles, s.info, s.b = tiles.data_ptr(), info.data_ptr(), b.data_ptr()
    rel, r2, b2 = C.c_double(), C.c_double(), C.c_double()
    st = _NA["poisson_residual_noalloc"](C.byref(s), C.c_void_p(x.data_ptr()), C.c_void_p(int(stream)), C.byref(rel), C.byref(r2), C.byref(b2))
    if st != abi.ST_OK:
        raise status_error("poisson residual_noalloc", st)
    return rel.value, r2.value, b2.value
