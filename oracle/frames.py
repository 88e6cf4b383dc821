"""CPU restatement of the frame packing and the bake measurements, test infrastructure only: the checker that the
device frame (st_flip_read_frame) and measurements (st_flip_bake_diag) are compared with.

pack_frame_buf follows packFrameBuf (src/gpu.js:525-560) for the water points of a particle readback, in the
reference's JavaScript double arithmetic: Math.round (nearest, halves up), a Uint8Array store (truncation), the frame
cut after the last live point. bake_diag follows bakeDiag (src/flip/bake.js:60-83)."""
import numpy as np


def js_round(v):
    r = np.floor(v)
    return r + (v - r >= 0.5)


def pack_frame_buf(buf, n, box, vs=1.0):
    """buf: (>= n, 4) float32 positions in id order (readbackInto); box: (x0, y0, z0, x1, y1, z1) as doubles."""
    b = np.asarray(buf[:n], np.float32)
    U = b.view(np.uint32)
    x, y, z, w = (b[:, k].astype(np.float64) for k in range(4))
    ks = 16.0 * (vs or 1.0)
    water = ~(y <= -1e5) & ~(U[:, 3] >= 0x80000000) & ~(w >= 4096)
    idx = np.nonzero(water)[0]
    m = int(idx[-1]) + 1 if len(idx) else 0
    x0, y0, z0, x1, y1, z1 = box
    k3 = (65535.0 / (x1 - x0), 65535.0 / (y1 - y0), 65535.0 / (z1 - z0))
    pos = np.zeros((m, 3), np.uint16)
    spd = np.zeros(m, np.uint8)
    fm = np.zeros(m, np.uint8)
    gone = y[:m] < -1e5
    other = (U[:m, 3] >= 0x80000000) | (w[:m] >= 4096)
    ok = ~gone & ~other
    for a, (c, lo) in enumerate(((x, x0), (y, y0), (z, z0))):
        q = js_round((c[:m] - lo) * k3[a])
        pos[ok, a] = np.clip(q, 0, 65535)[ok].astype(np.uint16)
    lv = np.floor(w[:m] / 64.0)
    s = (w[:m] - lv * 64.0) * ks
    sv = np.where(s > 191, 191.0, np.trunc(s))
    spd[:] = 255
    spd[ok] = (sv[ok].astype(np.int64) % 256).astype(np.uint8)
    fm[ok & (lv != 0)] = (lv[ok & (lv != 0)] * 17).astype(np.int64).astype(np.uint8)
    any_foam = bool(np.any(ok & (lv != 0)))
    return dict(n=m, pos=pos, spd=spd, fm=fm if any_foam else None)


def bake_diag(dst, n, box, vcap=14.0):
    H = 16
    x0, y0, z0, x1, y1, z1 = box
    hy = (y1 - y0) / H
    cap = min(vcap or 14, 63) * 0.98
    e = 1e-3
    d = np.asarray(dst[:n], np.float32).astype(np.float64)
    fin = np.all(np.isfinite(d), axis=1)
    bad = int((~fin).sum())
    live = fin & ~(d[:, 1] < -1e5)
    a = d[live]
    alive = len(a)
    x, y, z, w = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    lv = np.floor(w / 64)
    sp = w - lv * 64
    out = int(((x < x0 - e) | (x > x1 + e) | (y < y0 - e) | (y > y1 + e) | (z < z0 - e) | (z > z1 + e)).sum())
    hist = np.bincount(np.clip(np.floor((y - y0) / hy), 0, H - 1).astype(np.int64), minlength=H)
    k = max(alive, 1)
    return dict(alive=alive, gone=n - alive - bad, nonFinite=bad, outsideBox=out, atWaterSpeedLimit=int((sp >= cap).sum()),
                meanSpeed=float(sp.sum() / k), maxSpeed=float(sp.max()) if alive else 0.0, meanFoam=float(lv.sum() / k / 15),
                foamyPoints=int((lv >= 8).sum()), center=[float(x.sum() / k), float(y.sum() / k), float(z.sum() / k)],
                bbox=[float(x.min()), float(y.min()), float(z.min()), float(x.max()), float(y.max()), float(z.max())] if alive else None,
                heightHist=[int(v) for v in hist])
