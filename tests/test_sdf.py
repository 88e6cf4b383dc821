"""Mesh colliders: the signed distance grid of buildSDF (src/shared.js:98-181).

CPU: the oracle (oracle/sdf_oracle.cpp, the reference's passes in its order) against known answers: the grid's size
rule, exact distances near a box's faces, the sign everywhere, the chamfer distances within a few percent far out.
GPU: st_build_sdf equals the oracle bit for bit (its chamfer sweeps run as diagonal wavefronts; the exact band with
atomic minima)."""
import math

import numpy as np
import pytest


def uv_sphere(r, seg=14, rings=9):
    """A closed sphere of quads with triangle fans at the poles, wound outwards."""
    v = [[0.0, -r, 0.0]]
    for i in range(1, rings):
        a = -math.pi / 2 + i / rings * math.pi
        for j in range(seg):
            b = j / seg * 2 * math.pi
            v.append([math.cos(b) * math.cos(a) * r, math.sin(a) * r, math.sin(b) * math.cos(a) * r])
    v.append([0.0, r, 0.0])
    ring = lambda i, j: 1 + (i - 1) * seg + (j + seg) % seg   # noqa: E731
    f = [[0, ring(1, j + 1), ring(1, j)] for j in range(seg)]
    f += [[ring(i, j), ring(i, j + 1), ring(i + 1, j + 1), ring(i + 1, j)] for i in range(1, rings - 1) for j in range(seg)]
    f += [[len(v) - 1, ring(rings - 1, j), ring(rings - 1, j + 1)] for j in range(seg)]
    return np.array(v), f


def box(hx, hy, hz, shift=(0.0, 0.0, 0.0)):
    v = np.array([[x * hx, y * hy, z * hz] for z in (-1, 1) for y in (-1, 1) for x in (-1, 1)]) + np.array(shift)
    f = [[0, 4, 6, 2], [1, 3, 7, 5], [0, 1, 5, 4], [2, 6, 7, 3], [0, 2, 3, 1], [4, 5, 7, 6]]
    return v, f


def torus(R, r, seg=24, sides=12):
    v = []
    for i in range(seg):
        a = i / seg * 2 * math.pi
        for j in range(sides):
            b = j / sides * 2 * math.pi
            v.append([(R + r * math.cos(b)) * math.cos(a), r * math.sin(b), (R + r * math.cos(b)) * math.sin(a)])
    idx = lambda i, j: (i % seg) * sides + (j % sides)   # noqa: E731
    f = [[idx(i, j), idx(i, j + 1), idx(i + 1, j + 1), idx(i + 1, j)] for i in range(seg) for j in range(sides)]
    return np.array(v), f


def coords(s):
    nx, ny, nz = s["dims"]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    o, c = s["origin"], s["cell"]
    return o[0] + i * c, o[1] + j * c, o[2] + k * c


def test_box_distances_signs_and_grid():
    from oracle.oracle import build_sdf
    s = build_sdf(*box(0.2, 0.1, 0.15), cell=0.02, margin=0.1)
    # the grid: bounds grown by the margin, ceil(extent / cell) + 1 voxels per axis, in doubles (0.2 + 0.1 is
    # 0.30000000000000004, so the x extent over 0.02 is just above 30 and rounds up to 31)
    h = (0.2, 0.1, 0.15)
    assert s["dims"] == [math.ceil(((x + 0.1) - (-x - 0.1)) / 0.02) + 1 for x in h] == [32, 21, 26]
    assert s["origin"] == [-x - 0.1 for x in h]
    X, Y, Z = coords(s)
    d = s["data"].reshape(X.shape)
    qx, qy, qz = np.abs(X) - 0.2, np.abs(Y) - 0.1, np.abs(Z) - 0.15
    out = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2 + np.maximum(qz, 0) ** 2)
    ref = out + np.minimum(np.maximum(qx, np.maximum(qy, qz)), 0)
    near = np.abs(ref) <= 2.4 * s["cell"]
    assert np.abs(d - ref)[near].max() < 1e-6                 # exact band (f32 rounding)
    assert np.all(np.sign(d)[np.abs(ref) > 1e-3] == np.sign(ref)[np.abs(ref) > 1e-3])
    far = np.abs(ref) > 2.6 * s["cell"]
    assert np.all(np.abs(d - ref)[far] <= 0.1 * np.abs(ref)[far] + 1e-6)   # chamfer: within a few percent


def test_sphere_and_the_voxel_cap():
    from oracle.oracle import build_sdf
    v, f = uv_sphere(0.3, 24, 16)
    s = build_sdf(v, f, cell=0.02)
    X, Y, Z = coords(s)
    ref = np.sqrt(X ** 2 + Y ** 2 + Z ** 2) - 0.3
    d = s["data"].reshape(X.shape)
    assert np.abs(d - ref)[np.abs(ref) < 0.04].max() < 0.005   # faceting of 24 x 16 quads
    assert np.all((d < 0) == (ref < 0)) or np.all(((d < 0) != (ref < 0)) <= (np.abs(ref) < 0.005))
    big = build_sdf(v, f, cell=0.002)                         # 382^3 voxels: the cell grows by 1.25 until <= 2.6M
    lo, hi = v.min(0) - 0.16, v.max(0) + 0.16
    count = lambda c: np.prod([math.ceil((hi[k] - lo[k]) / c) + 1 for k in range(3)])   # noqa: E731
    assert count(big["cell"]) <= 2.6e6 < count(big["cell"] / 1.25) and big["cell"] > 0.002


def test_degenerate_meshes():
    """No vertices: the reference's grid size is negative (a RangeError); here a BAD_ARG error. A mesh of faces with
    no area (a flat quad seen along y) still gets exact distances, and no voxel is inside."""
    from oracle.oracle import build_sdf
    from splashtank_b200.flip import StError
    with pytest.raises(StError):
        build_sdf(np.zeros((0, 3)), [], cell=0.5, margin=0.0)
    v = np.array([[0.0, 0.0, 0.0], [0.2, 0.0, 0.0], [0.2, 0.0, 0.2], [0.0, 0.0, 0.2]])
    s = build_sdf(v, [[0, 1, 2, 3]], cell=0.05, margin=0.1)
    assert (s["data"] >= 0).all() and s["data"].min() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["sphere", "box", "torus", "shifted_box_fine"])
def test_device_builder_matches_the_oracle(shape):
    from oracle.oracle import build_sdf as oracle_sdf
    from splashtank_b200.sdf import build_sdf
    mesh, kw = {"sphere": (uv_sphere(0.3, 24, 16), dict(cell=0.02)), "box": (box(0.2, 0.1, 0.15), dict(cell=0.02, margin=0.1)),
                "torus": (torus(0.35, 0.1), dict(cell=0.015)),
                "shifted_box_fine": (box(0.31, 0.22, 0.4, (0.13, -0.05, 0.2)), dict(cell=0.004))}[shape]
    got, want = build_sdf(*mesh, **kw), oracle_sdf(*mesh, **kw)
    assert got["dims"] == want["dims"] and got["origin"] == want["origin"] and got["cell"] == want["cell"]
    assert np.array_equal(got["data"].view(np.uint32), want["data"].view(np.uint32))
    assert (got["data"] < 0).any() and (got["data"] > 0).any()
