"""Signed distance grids of closed meshes (buildSDF, src/shared.js:98-181), built on the GPU by st_build_sdf.

The result is the reference's sdf object: id, dims, origin, cell, data (float32, x fastest, negative inside), ready to
be a collider's grid (st_sdf).
"""
import ctypes as C
import itertools

import numpy as np

from . import abi
from .flip import load_library, status_error

_F = None
_IDS = itertools.count(1)   # SDF_ID (src/shared.js:8)


def funcs():
    global _F
    if _F is None:
        _F = abi.bind(load_library()[0], "st_", abi.SDF_FUNCS)
    return _F


def mesh_struct(v, faces):
    """v: (nv, 3) vertex positions; faces: polygons as sequences of vertex indices. Returns (st_mesh, keepalive)."""
    v = np.ascontiguousarray(np.asarray(v, np.float64).reshape(-1, 3))
    idx = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in faces]) if len(faces) else np.zeros(0, np.uint32))
    ln = np.ascontiguousarray(np.array([len(f) for f in faces], np.uint32))
    m = abi.Mesh()
    m.v = v.ctypes.data_as(C.POINTER(C.c_double))
    m.nv = len(v)
    m.idx = idx.ctypes.data_as(abi.u32p)
    m.len = ln.ctypes.data_as(abi.u32p)
    m.nf = len(ln)
    return m, (v, idx, ln)


def build_sdf(v, faces, cell=0.025, margin=0.16, device=0, fn=None):
    """buildSDF(mesh, cell, margin): dict(id, dims, origin, cell, data). fn: an entry point with st_build_sdf's
    arguments after the device (defaults to the GPU builder)."""
    m, keep = mesh_struct(v, faces)
    b = abi.SdfBuild()
    b.size = C.sizeof(abi.SdfBuild)
    b.cell = float(cell)
    b.margin = float(margin)
    call = fn or (lambda mp, bp: funcs()["build_sdf"](int(device), mp, bp))
    st = call(C.byref(m), C.byref(b))
    if st != abi.ST_OK:
        raise status_error("build_sdf", st)
    dims = [int(x) for x in b.dims]
    data = np.zeros(dims[0] * dims[1] * dims[2], np.float32)
    b.data = data.ctypes.data_as(abi.f32p)
    b.cap = len(data)
    st = call(C.byref(m), C.byref(b))
    if st != abi.ST_OK:
        raise status_error("build_sdf", st)
    del keep
    return dict(id=next(_IDS), dims=dims, origin=[float(x) for x in b.origin], cell=float(b.cell), data=data)
