"""Differentiable FLIP rollout (st_diff_*): forward loss and the hand-written adjoint's gradient with respect to 8
collider keyframes and the initial fluid velocity. Compute runs in libsplashtank_cuda.so."""
import ctypes as C

import numpy as np

from . import abi
from .flip import load_library, status_error

_D = None
NPARAM = 27


def funcs():
    global _D
    if _D is None:
        _D = abi.bind(load_library()[0], "st_", abi.DIFF_FUNCS)
    return _D


class DiffRollout:
    def __init__(self, n, pos, target, steps, ckpt_every=8, fp64=False, dt=1.0 / 240.0, flip=0.95, g=9.81, q0=None,
                 margin=None, box_half=(0.06, 0.12, 0.25), cg_maxit=None, cg_tol=None, device=0, collider="box", grid_cell=None):
        """collider: "box" (analytic signed distance) or "grid" (the box's distance grid with nodes grid_cell apart,
        default half a cell, sampled and differentiated as sdfEval samples a collider grid)."""
        self.f = funcs()
        d = abi.DiffDesc()
        d.size = C.sizeof(abi.DiffDesc)
        d.n, d.steps, d.ckpt_every, d.fp64, d.device = int(n), int(steps), int(ckpt_every), 1 if fp64 else 0, int(device)
        h = 1.0 / n
        d.dt, d.flip, d.g = float(dt), float(flip), float(g)
        d.q0 = float(q0 if q0 is not None else 0.3 * h)
        d.margin = float(margin if margin is not None else 0.5 * h)
        d.box_half[:] = [float(x) for x in box_half]
        d.cg_maxit = int(cg_maxit if cg_maxit is not None else (4000 if fp64 else 1000))
        d.cg_tol = float(cg_tol if cg_tol is not None else (1e-12 if fp64 else 1e-5))
        d.collider_grid = 1 if collider == "grid" else 0
        d.grid_cell = float(grid_cell if grid_cell is not None else 0.5 * h)
        p = np.ascontiguousarray(pos, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        assert t.size == n ** 3
        h_ = C.c_void_p()
        st = self.f["diff_create"](C.byref(d), p.ctypes.data_as(abi.f32p), len(p), t.ctypes.data_as(abi.f32p), C.byref(h_))
        if st != abi.ST_OK:
            raise status_error("diff create", st)
        self._h = h_
        self.n, self.steps, self.np = n, steps, len(p)

    def forward(self, params, record=True):
        prm = np.ascontiguousarray(params, np.float64)
        assert prm.size == NPARAM
        loss = C.c_double()
        st = self.f["diff_forward"](self._h, prm.ctypes.data_as(C.POINTER(C.c_double)), 1 if record else 0, C.byref(loss))
        if st != abi.ST_OK:
            raise status_error("diff forward", st)
        return loss.value

    def backward(self):
        g = np.zeros(NPARAM, np.float64)
        st = self.f["diff_backward"](self._h, g.ctypes.data_as(C.POINTER(C.c_double)))
        if st != abi.ST_OK:
            raise status_error("diff backward", st)
        return g

    def state(self):
        """(positions, velocities) of the particles after the last forward pass, (np, 3) float32 each."""
        p = np.zeros((self.np, 3), np.float32)
        v = np.zeros((self.np, 3), np.float32)
        st = self.f["diff_read_state"](self._h, p.ctypes.data_as(abi.f32p), v.ctypes.data_as(abi.f32p))
        if st != abi.ST_OK:
            raise status_error("diff read_state", st)
        return p, v

    def stream(self):
        return self.f["diff_stream"](self._h)

    def stats(self):
        b, it = C.c_uint64(), C.c_int32()
        self.f["diff_stats"](self._h, C.byref(b), C.byref(it))
        return b.value, it.value

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["diff_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def flip_rollout(dam, params, box_half=(0.06, 0.12, 0.25), iters=400, omega=1.9, device=0):
    """The same rollout through the FLIP step itself (st_flip_step): dam's particles (unit box, shifted into the
    reference box) with the initial velocity params[24:27], the box collider as its distance grid (half a cell apart)
    moving along the keyframe path params[:24] (linear, keyframes evenly over the rollout, the collider's velocity from
    consecutive poses as SceneRunner gives it), FLIP 0.95, gravity 9.81, no density correction, no sheet tearing, the
    SOR run for `iters` iterations. Returns the particles' final positions in the unit box, in the input order."""
    from .flip import FlipSim
    from .scene import SceneRunner, box_sdf
    n, steps = dam.n, dam.steps
    h = 1.0 / n
    sim = FlipSim(h / 2, len(dam.pos), size=(1.0, 1.0, 1.0), device=device)
    p0 = dam.pos.astype(np.float32).copy()
    p0[:, 0] -= 0.5
    p0[:, 2] -= 0.5
    sim.add_many(p0, np.tile(np.asarray(params[24:27], np.float32)[None, :], (len(p0), 1)))
    sdf = box_sdf(*box_half, h / 2, sid=1)
    K = np.asarray(params[:24], np.float64).reshape(8, 3)
    T = steps / 240.0

    def centre(t):
        u = t / T * 7.0
        i = min(6, max(0, int(np.floor(u))))
        a = u - i
        return (1 - a) * K[i] + a * K[i + 1]
    run = SceneRunner(sim)
    opts = dict(g=9.81, flip=0.95, comp=0.0, iters=iters, omega=omega, vmax=100.0, tear=0.0)
    for k in range(steps):
        c = centre((k + 1) / 240.0)
        run.step(1 / 240.0, [dict(id=1, sdf=sdf, x=c[0] - 0.5, y=c[1], z=c[2] - 0.5)], opts)
    out = np.zeros((len(p0), 4), np.float32)
    sim.readbackInto(out)
    sim.destroy()
    x = out[:, :3].copy()
    x[:, 0] += 0.5
    x[:, 2] += 0.5
    return x
