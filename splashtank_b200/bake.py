"""The bake loop around the step (runBakeFlipGpu, src/flip/bake.js:85-132) and the cache file it fills
(writeCacheParts / parseCache2, src/shared.js:688-736).

Frames come from st_flip_read_frame (packed on the device in id order) and the per-frame measurements from
st_flip_bake_diag, so a frame costs 8 bytes per point of readback instead of a 16-byte float copy per point. The
whitewater part (packSprayFrame, st_flip_read_spray_frame) and, with the deep look on, the deep-water part (readDeep +
packDeep, st_flip_read_deep) are packed on the device too.
"""
import json
import math
import struct

import numpy as np


def obj_speed(a, b, dt, lim):
    """objSpeed (src/shared.js:512-524): the fastest object motion between two sampled states (emitters count by speed)."""
    v = 0.0
    for i, o in enumerate(b):
        p = a[i] if a and i < len(a) else None
        if o.get("kind") == "emitter":
            if o.get("on"):
                v = max(v, o.get("speed", 0.0))
            continue
        if not p or p.get("id") != o.get("id"):
            continue
        lin = math.hypot(o["x"] - p["x"], o["y"] - p["y"], o["z"] - p["z"])
        rot = abs(o.get("rx", 0) - p.get("rx", 0)) + abs(o.get("yaw", 0) - p.get("yaw", 0)) + abs(o.get("rz", 0) - p.get("rz", 0))
        sdf = o.get("sdf")
        R = 0.5 * sdf["cell"] * math.hypot(*sdf["dims"]) if sdf else 0.5
        ov = (lin + rot * R) / dt
        if not lim or ov <= lim:
            v = max(v, ov)
    return v


def pack_objs(states):
    """packObjs (src/shared.js:654-658): 6 floats per object."""
    out = np.zeros(len(states) * 6, np.float32)
    for k, o in enumerate(states):
        out[k * 6:k * 6 + 6] = [o["x"], o["y"], o["z"], o.get("rx", 0), o.get("yaw", 0), o.get("rz", 0)]
    return out


def run_bake(sim, runner, states, par, fps, frames, substeps=1, cfl=1.5, max_sub=16, vmax0=2.0, scale=1.0, on_frame=None, nb_look=False):
    """runBakeFlipGpu's frame loop (src/flip/bake.js:101-131) for a filled simulator: substeps per frame adapt to the
    fastest particle of the last frame and the objects' own motion; every frame is read as a packed frame with its
    measurements, plus its whitewater points (when the simulator has a pool) and deep-water points (nb_look).
    states(t) gives the objects; par the step options. Returns the list of frames."""
    if nb_look:
        sim.setDeepLook(True)
    foam_life = ((par.get("spr") or {}).get("ww") or {}).get("foamLife") or 3.0
    dtF = 1.0 / fps
    max_sub = max(substeps, max_sub)
    out = []

    def frame(f, sub, objv):
        fr = sim.read_frame(scale)
        fr["objs"] = pack_objs(states(f * dtF))
        diag = sim.bake_diag(par.get("vmax", 14.0))
        diag.update(sub=sub, objectSpeed=objv)
        if f > 0 and sim.sprayCap:
            fr["sp"] = sim.read_spray_frame(200000, foam_life)
            diag["sprayPoints"] = fr["sp"]["alive"]
        if f > 0 and nb_look:
            dp = sim.read_deep(scale)
            if dp:
                fr["dp"] = dp
                diag["deepPoints"] = dp["n"]
        if on_frame:
            on_frame(fr, dict(f=f, F=frames, n=fr["n"], sub=sub, diag=diag))
        out.append((fr, diag))
        return diag

    vmax = vmax0
    frame(0, 0, 0.0)
    for f in range(1, frames + 1):
        objv = obj_speed(states((f - 1) * dtF), states(f * dtF), dtF, par.get("colMax", 20.0))
        sub = max(substeps, min(max_sub, math.ceil(dtF * max(vmax, objv) / (cfl * sim.h))))
        dt = dtF / sub
        for s in range(sub):
            t = (f - 1) * dtF + (s + 1) * dt
            o = dict(par)
            o["time"] = t
            runner.step(dt, states(t), o)
        diag = frame(f, sub, objv)
        st = sim.readStats()
        vmax = max(1.0, diag["maxSpeed"] or 0.0, st["vmax"])
    return out


def write_cache(frames, meta):
    """writeCacheParts (src/shared.js:688-705), version 2: 'SPLC', 2, the JSON block, padding, frame count, then per
    frame: points, flags (1 = white-water bytes follow, 2 = whitewater points follow, 4 = deep-water points follow),
    object poses, positions, speeds, [white water], padding, [whitewater: count, positions, padding, codes], [deep
    water: count, positions, speeds, padding]."""
    mj = json.dumps(meta, separators=(",", ":")).encode()
    pad = lambda k: b"\0" * ((4 - k % 4) % 4)   # noqa: E731
    parts = [b"SPLC", struct.pack("<II", 2, len(mj)), mj, pad(len(mj)), struct.pack("<I", len(frames))]
    for fr in frames:
        n, fm = fr["n"], fr.get("fm")
        sp = fr.get("sp") if fr.get("sp") and fr["sp"]["n"] else None
        dp = fr.get("dp") if fr.get("dp") and fr["dp"]["n"] else None
        parts.append(struct.pack("<II", n, (1 if fm is not None else 0) | (2 if sp else 0) | (4 if dp else 0)))
        parts.append(np.asarray(fr["objs"], np.float32).tobytes())
        parts.append(np.asarray(fr["pos"], np.uint16).tobytes())
        parts.append(np.asarray(fr["spd"], np.uint8).tobytes())
        nb = n * 7
        if fm is not None:
            parts.append(np.asarray(fm, np.uint8).tobytes())
            nb += n
        parts.append(pad(nb))
        if sp:
            parts += [struct.pack("<I", sp["n"]), np.asarray(sp["pos"], np.uint16).tobytes(), pad(sp["n"] * 6),
                      np.asarray(sp["pk"], np.uint32).tobytes()]
        if dp:
            parts += [struct.pack("<I", dp["n"]), np.asarray(dp["pos"], np.uint16).tobytes(), np.asarray(dp["spd"], np.uint8).tobytes(),
                      pad(dp["n"] * 7)]
    return b"".join(parts)


def parse_cache(buf):
    """parseCache2 (src/shared.js:706-736): (meta, frames), frames with their whitewater (sp) and deep-water (dp) parts."""
    assert buf[:4] == b"SPLC" and struct.unpack_from("<I", buf, 4)[0] == 2
    ml = struct.unpack_from("<I", buf, 8)[0]
    o = 12
    meta = json.loads(buf[o:o + ml].decode())
    o += ml + (4 - ml % 4) % 4
    nf = struct.unpack_from("<I", buf, o)[0]
    o += 4
    nobj = len(meta.get("ids", []))
    frames = []
    for _ in range(nf):
        n, fl = struct.unpack_from("<II", buf, o)
        o += 8
        objs = np.frombuffer(buf, np.float32, nobj * 6, o)
        o += nobj * 24
        pos = np.frombuffer(buf, np.uint16, n * 3, o).reshape(n, 3)
        o += n * 6
        spd = np.frombuffer(buf, np.uint8, n, o)
        o += n
        fm = None
        if fl & 1:
            fm = np.frombuffer(buf, np.uint8, n, o)
            o += n
        o += (4 - (n * (8 if fl & 1 else 7)) % 4) % 4
        fr = dict(n=n, pos=pos, spd=spd, fm=fm, objs=objs)
        if fl & 2:
            ns = struct.unpack_from("<I", buf, o)[0]
            o += 4
            p2 = np.frombuffer(buf, np.uint16, ns * 3, o).reshape(ns, 3)
            o += ns * 6 + (4 - ns * 6 % 4) % 4
            pk = np.frombuffer(buf, np.uint32, ns, o)
            o += ns * 4
            fr["sp"] = dict(n=ns, pos=p2, pk=pk, alive=ns)
        if fl & 4:
            nd = struct.unpack_from("<I", buf, o)[0]
            o += 4
            p3 = np.frombuffer(buf, np.uint16, nd * 3, o).reshape(nd, 3)
            o += nd * 6
            s3 = np.frombuffer(buf, np.uint8, nd, o)
            o += nd + (4 - nd * 7 % 4) % 4
            fr["dp"] = dict(n=nd, pos=p3, spd=s3)
        frames.append(fr)
    return meta, frames
