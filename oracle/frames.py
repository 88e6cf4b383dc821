"""CPU restatement of the frame packing and the bake measurements, test infrastructure only: the checker that the
device frame (st_flip_read_frame) and measurements (st_flip_bake_diag) are compared with.

pack_frame_buf follows packFrameBuf (src/gpu.js:525-560) for the water points of a particle readback, in the
reference's JavaScript double arithmetic: Math.round (nearest, halves up), a Uint8Array store (truncation), the frame
cut after the last live point. bake_diag follows bakeDiag (src/flip/bake.js:60-83). pack_spray_frame and pack_deep
follow packSprayFrame / packSprayJS (src/flip/bake.js:4-15, 43-58) and packDeep (src/gpu.js:512-524), also in
doubles; pack_live follows the live view's packDisp, sprayDisp and packSpray (src/flip/wgsl-whitewater.js:183-253) in
the shader's f32 arithmetic. Math.hypot is taken as the square root of the sum of squares."""
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


# ---- JavaScript number helpers (float64 arrays) ----
def js_int32(x):
    """ToInt32: NaN and infinities give 0, the rest is truncated modulo 2^32 (as uint32 bits)."""
    x = np.asarray(x, np.float64)
    ok = np.isfinite(x)
    t = np.where(ok, np.trunc(np.where(ok, x, 0.0)), 0.0)
    return np.mod(t, 4294967296.0).astype(np.uint64).astype(np.uint32)


def q16_js(v, lo, k):
    return np.clip(js_round((np.asarray(v, np.float64) - lo) * k), 0, 65535).astype(np.uint16)


def pack_spray_js(v, kind_rounded, life_frac):
    """packSprayJS (src/flip/bake.js:4-15) for arrays: v (n, 3) float64, kind_rounded Math.round of the kind word."""
    with np.errstate(all="ignore"):
        vx, vy, vz = (np.asarray(v[:, a], np.float64) for a in range(3))
        kind = js_int32(kind_rounded).view(np.int32)
        sp = np.sqrt(vx * vx + vy * vy + vz * vz)
        code = np.uint32(0x80000000) | (js_int32(np.minimum(np.floor(sp * 4.0), 255.0)) << np.uint32(21))
        kb = np.array([0, 0x40000000, 0x20000000, 0x60000000], np.uint32)
        code = code | kb[kind & 3]
        lf = np.asarray(life_frac, np.float64)
        lf = np.where(np.isnan(lf) | (lf == 0), 0.0, lf)
        foam = code | js_int32(js_round(np.maximum(0.0, np.minimum(1.0, lf)) * 1023.0))
        big = sp > 1e-6
        nx = np.where(big, vx / sp, 0.0)
        ny = np.where(big, vy / sp, 1.0)
        nz = np.where(big, vz / sp, 0.0)
        l = np.abs(nx) + np.abs(ny) + np.abs(nz)
        px, py = nx / l, ny / l
        neg = nz < 0
        qx = (1.0 - np.abs(py)) * np.where(px >= 0, 1.0, -1.0)
        qy = (1.0 - np.abs(px)) * np.where(py >= 0, 1.0, -1.0)
        px, py = np.where(neg, qx, px), np.where(neg, qy, py)
        u = js_int32(np.maximum(0.0, np.minimum(1023.0, js_round((px * 0.5 + 0.5) * 1023.0))))
        w = js_int32(np.maximum(0.0, np.minimum(1023.0, js_round((py * 0.5 + 0.5) * 1023.0))))
        return np.where(kind >= 2, foam, code | (w << np.uint32(10)) | u).astype(np.uint32)


def pack_spray_frame(sp, sv, n, box, cap, foam_life):
    """packSprayFrame (src/flip/bake.js:43-58): sp, sv (>= n, 4) float32 slots of readSpray."""
    foam_life = foam_life or 3.0
    p = np.asarray(sp[:n], np.float32)
    alive_m = p[:, 3] > 0
    alive = int(alive_m.sum())
    step = max(1, int(np.ceil(alive / cap)))
    j = np.arange(0, n, step)
    j = j[alive_m[j]]
    x0, y0, z0, x1, y1, z1 = box
    k3 = (65535.0 / (x1 - x0), 65535.0 / (y1 - y0), 65535.0 / (z1 - z0))
    pd = p[j].astype(np.float64)
    vd = np.asarray(sv, np.float32)[j].astype(np.float64)
    pos = np.stack([q16_js(pd[:, 0], x0, k3[0]), q16_js(pd[:, 1], y0, k3[1]), q16_js(pd[:, 2], z0, k3[2])], 1)
    pk = pack_spray_js(vd[:, :3], js_round(vd[:, 3]), pd[:, 3] / foam_life)
    return dict(n=len(j), pos=pos, pk=pk, alive=alive)


def pack_deep(points, box, vs=1.0):
    """packDeep (src/gpu.js:512-524): points (n, 4) float32 (x, y, z, 4096 + speed)."""
    p = np.asarray(points, np.float32).astype(np.float64)
    p = p[~(p[:, 1] <= -1e5)]
    x0, y0, z0, x1, y1, z1 = box
    k3 = (65535.0 / (x1 - x0), 65535.0 / (y1 - y0), 65535.0 / (z1 - z0))
    pos = np.stack([q16_js(p[:, 0], x0, k3[0]), q16_js(p[:, 1], y0, k3[1]), q16_js(p[:, 2], z0, k3[2])], 1)
    with np.errstate(all="ignore"):
        s = (p[:, 3] - 4096.0) * (16.0 * (vs or 1.0))
        spd = np.where(s > 191, 191, js_int32(np.maximum(0.0, s)) & 0xff).astype(np.uint8)
    return dict(n=len(p), pos=pos, spd=spd)


# ---- the live view in f32 (packDisp) ----
F32 = np.float32


def _fmx(a, b):
    return np.where(a > b, a, b)


def _fmn(a, b):
    return np.where(a < b, a, b)


def _clampf(x, lo, hi):
    return _fmn(_fmx(x, F32(lo)), F32(hi)).astype(np.float32)


def _u32f(f):
    f = np.asarray(f, np.float32)
    with np.errstate(all="ignore"):
        t = np.where(np.isnan(f) | (f <= 0), 0.0, np.minimum(np.trunc(f.astype(np.float64)), 4294967295.0))
    return t.astype(np.uint64).astype(np.uint32)


def _q16f(v, lo, k):
    return _u32f(_clampf(np.rint((np.asarray(v, np.float32) - F32(lo)) * F32(k)).astype(np.float32), 0.0, 65535.0)).astype(np.uint16)


def pack_spray_f32(v, kind, life_frac):
    """packSpray (src/flip/wgsl-whitewater.js:183-193) in f32: v (n, 3) float32, kind (n,) uint32."""
    with np.errstate(all="ignore"):
        v = np.asarray(v, np.float32)
        s = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]).astype(np.float32)
        code = np.uint32(0x80000000) | (np.minimum(_u32f(s * F32(4.0)), np.uint32(255)) << np.uint32(21))
        code = code | np.select([kind == 1, kind == 2, kind == 3], [0x40000000, 0x20000000, 0x60000000], 0).astype(np.uint32)
        foam = code | _u32f(_clampf(np.asarray(life_frac, np.float32), 0.0, 1.0) * F32(1023.0))
        big = s > F32(1e-6)
        n = np.where(big[:, None], v / np.where(big, s, F32(1.0))[:, None], np.array([0, 1, 0], np.float32)).astype(np.float32)
        l = ((np.abs(n[:, 0]) + np.abs(n[:, 1])) + np.abs(n[:, 2])).astype(np.float32)
        px, py = (n[:, 0] / l).astype(np.float32), (n[:, 1] / l).astype(np.float32)
        neg = n[:, 2] < 0
        qx = ((F32(1.0) - np.abs(py)) * np.where(px >= 0, F32(1.0), F32(-1.0))).astype(np.float32)
        qy = ((F32(1.0) - np.abs(px)) * np.where(py >= 0, F32(1.0), F32(-1.0))).astype(np.float32)
        px, py = np.where(neg, qx, px), np.where(neg, qy, py)
        u = _u32f(_clampf(np.rint((px * F32(0.5) + F32(0.5)) * F32(1023.0)).astype(np.float32), 0.0, 1023.0))
        w = _u32f(_clampf(np.rint((py * F32(0.5) + F32(0.5)) * F32(1023.0)).astype(np.float32), 0.0, 1023.0))
        return np.where(kind >= 2, foam, code | (w << np.uint32(10)) | u).astype(np.uint32)


def pack_live(layout, pos_storage, stride, s_pos, s_vel, used, sd_max, foam_life, deep, box, vs=1.0):
    """The packed live view (packDisp with subsample and sprayDisp, src/flip/wgsl-whitewater.js:196-253,
    src/flip/wgsl-solver.js:141-147): layout as st_live_layout fields; pos_storage (N, 4) float32 positions in storage
    order; s_pos, s_vel the whitewater slots; used the slots handed out (min(sctl[0], smax)); deep the deep points."""
    L = layout
    out = np.zeros(L["words"], np.uint32)
    x0, y0, z0, x1, y1, z1 = box
    k3 = (F32(65535.0 / (x1 - x0)), F32(65535.0 / (y1 - y0)), F32(65535.0 / (z1 - z0)))
    o3 = (F32(x0), F32(y0), F32(z0))
    vsf = F32(vs or 1.0)
    u8 = out.view(np.uint8)
    u16 = out.view(np.uint16)
    # water
    nW = L["n_water"]
    n4 = (nW + 3) // 4 * 4
    v = np.tile(np.array([0.0, -1.0e6, 0.0, 0.0], np.float32), (n4, 1))
    idx = np.arange(nW) * (1 if L["from_pos"] else stride)
    v[:nW] = np.asarray(pos_storage, np.float32)[idx]
    ok = v[:, 1] > F32(-1.0e5)
    q = np.zeros((n4, 3), np.uint16)
    for a in range(3):
        q[ok, a] = _q16f(v[ok, a], o3[a], k3[a])
    lv = np.floor(v[:, 3] / F32(64.0)).astype(np.float32)
    s = np.where(ok, _u32f(_clampf(((v[:, 3] - lv * F32(64.0)) * F32(16.0)) * vsf, 0.0, 191.0)), 255)
    f = np.where(ok, _u32f(_clampf(lv, 0.0, 15.0)) * 17, 0)
    u16[L["o_wp"] * 2: L["o_wp"] * 2 + n4 * 3] = q.ravel()
    u8[L["o_ws"] * 4: L["o_ws"] * 4 + n4] = s.astype(np.uint8)
    u8[L["o_wf"] * 4: L["o_wf"] * 4 + n4] = f.astype(np.uint8)
    # whitewater: every stride-th slot handed out, the living ones in slot order
    nS = 0
    if L["n_spray"] and sd_max:
        st = max(1, (used + sd_max - 1) // sd_max)
        j = np.arange(sd_max, dtype=np.int64) * st
        j = j[j < used]
        j = j[np.asarray(s_pos, np.float32)[j, 3] > 0]
        nS = len(j)
        p = np.asarray(s_pos, np.float32)[j]
        vv = np.asarray(s_vel, np.float32)[j]
        qs = np.stack([_q16f(p[:, a], o3[a], k3[a]) for a in range(3)], 1) if nS else np.zeros((0, 3), np.uint16)
        code = pack_spray_f32(vv[:, :3], _u32f(vv[:, 3] + F32(0.5)), p[:, 3] / _fmx(F32(foam_life), F32(0.01)))
        u16[L["o_sp"] * 2: L["o_sp"] * 2 + nS * 3] = qs.ravel()
        out[L["o_sk"]: L["o_sk"] + nS] = code
    # deep water
    nD = 0
    if L["n_deep"]:
        u8[L["o_ds"] * 4:] = 255
        if deep is not None:
            d = np.asarray(deep, np.float32)
            nD = len(d)
            okd = d[:, 1] > F32(-1.0e5)
            qd = np.zeros((nD, 3), np.uint16)
            for a in range(3):
                qd[okd, a] = _q16f(d[okd, a], o3[a], k3[a])
            sd = np.where(okd, _u32f(_clampf(((d[:, 3] - F32(4096.0)) * F32(16.0)) * vsf, 0.0, 191.0)), 255)
            u16[L["o_dp"] * 2: L["o_dp"] * 2 + nD * 3] = qd.ravel()
            u8[L["o_ds"] * 4: L["o_ds"] * 4 + nD] = sd.astype(np.uint8)
    out[0], out[1] = nS, nD
    return out
