"""Generates the golden fixtures of tests/golden from the oracle (python tests/golden/make_golden.py).

The reference's own tests hold no numerical fixtures for the FLIP step (its tests are browser scripts that only
check that the page steps), so these fixtures pin the oracle against regressions and give the GPU parity tests a
fixed target: the state after a few steps of two small seeded scenes, in storage order, plus the grid fields.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def run_case(name, cls=None):
    from splashtank_b200 import scenes
    from splashtank_b200.scene import SceneRunner
    if cls is None:
        from oracle.oracle import OracleFlipSim as cls
    kw = {"threads": 4} if cls.__name__.startswith("Oracle") else {}
    if name.startswith("dam_break"):
        n, steps = 16, 10
        sc = scenes.dam_break(n)
        s = cls(sc["d"], len(sc["pos"]), size=sc["size"], ratio=sc["ratio"], **kw)
        s.add_many(sc["pos"], sc["vel"])
        for _ in range(steps):
            s.step(sc["dt"], sc["opts"])
    else:
        w = scenes.WaveTank(24, spray_cap=20000)
        s = w.make(cls, **kw)
        r = SceneRunner(s)
        t = 0.0
        for _ in range(8):
            t += w.dt
            r.step(w.dt, w.states(t), w.opts)
    p, v, ids = s.save_state()
    g = s.grid()
    out = dict(pos=p, vel=v, ids=ids, tile_on=g["tile_on"], cnt=g["cnt"], ctype=g["ctype"], pres=g["pres"], vn=g["vn"], vo=g["vo"],
               velg=g["velg"])
    if getattr(s, "sprayCap", 0):
        sp = s.readSpray()
        out["spray_p"] = sp["p"]
        out["spray_v"] = sp["v"]
    return out


if __name__ == "__main__":
    for name in ("dam_break_16_s10", "wave_tank_24_s8"):
        out = run_case(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})
