"""Helpers shared by the parity tests: run the CUDA path and the CPU oracle on the same scene and compare."""
import numpy as np

from splashtank_b200 import scenes
from splashtank_b200.flip import FlipSim


def make_pair(sc, spray_cap=0, extra=1000):
    from oracle.oracle import OracleFlipSim
    n = len(sc["pos"])
    kw = dict(size=sc["size"], open=sc.get("open", 0), ratio=sc["ratio"], spray_cap=spray_cap)
    g = FlipSim(sc["d"], n + extra, **kw)
    o = OracleFlipSim(sc["d"], n + extra, threads=8, **kw)
    for s in (g, o):
        s.add_many(sc["pos"], sc["vel"])
    return g, o


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.sqrt(np.sum(b * b))
    num = np.sqrt(np.sum((a - b) ** 2))
    return float(num / den) if den > 0 else float(num)


def grid_report(g, o):
    """Compare the dense grid exports; returns dict of (exact, max abs diff) per field over cells with storage."""
    A, B = g.grid(), o.grid()
    out = {"tile_on": bool(np.array_equal(A["tile_on"], B["tile_on"]))}
    for k in ("cnt", "ctype"):
        out[k] = bool(np.array_equal(A[k], B[k]))
    for k in ("pres", "rhs", "vn", "vo", "velg"):
        a, b = A[k], B[k]
        out[k] = (bool(np.array_equal(a.view(np.uint32), b.view(np.uint32))), float(np.max(np.abs(a - b))) if a.size else 0.0,
                  rel_l2(a, b))
    return out, A, B


def state_report(g, o):
    pa, va, ia = g.save_state()
    pb, vb, ib = o.save_state()
    out = {"order": bool(np.array_equal(ia, ib))}
    out["pos_xyz_exact"] = bool(np.array_equal(pa[:, :3].view(np.uint32), pb[:, :3].view(np.uint32)))
    out["vel_xyz_exact"] = bool(np.array_equal(va[:, :3].view(np.uint32), vb[:, :3].view(np.uint32)))
    out["pos_xyz_maxdiff"] = float(np.max(np.abs(pa[:, :3] - pb[:, :3]))) if len(pa) else 0.0
    out["vel_xyz_maxdiff"] = float(np.max(np.abs(va[:, :3] - vb[:, :3]))) if len(va) else 0.0
    out["foam_maxdiff"] = float(np.max(np.abs(va[:, 3] - vb[:, 3]))) if len(va) else 0.0
    out["posw_mismatch"] = int(np.sum(pa[:, 3] != pb[:, 3]))
    return out
