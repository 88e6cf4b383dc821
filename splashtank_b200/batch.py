"""Many independent tanks stepped together (st_batch_*), the split of tanks over GPUs, and the launch-shape autotuner.

A batch step does every tank's FlipSim.step (src/flip/sim.js:179-241) with that tank's own options; the tanks' captured
step graphs run as parallel branches of one CUDA graph launch ("graph") or one after another ("sequential"), or the tanks
share one pool of fluid tiles for the pressure sweeps, swept for all tanks by one launch per colour ("pooled") or by one
persistent cooperative launch with bounded grid-barrier waits ("persistent"). Each tank gets exactly the result of
stepping it alone. Compute runs in libsplashtank_cuda.so.
"""
import ctypes as C
import time

from . import abi
from .flip import load_library, make_opts, status_error

_B = None


def funcs():
    global _B
    if _B is None:
        _B = abi.bind(load_library()[0], "st_", abi.BATCH_FUNCS)
    return _B


MODES = {"graph": abi.ST_BATCH_GRAPH, "sequential": abi.ST_BATCH_SEQUENTIAL, "pooled": abi.ST_BATCH_POOLED,
         "persistent": abi.ST_BATCH_PERSISTENT}


class TankBatch:
    """sims: FlipSim handles on one device (the caller keeps them alive and owns them)."""

    def __init__(self, sims, mode="graph"):
        self.f = funcs()
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s._h.value if hasattr(s._h, "value") else s._h for s in self.sims])
        d = abi.BatchDesc()
        d.size = C.sizeof(abi.BatchDesc)
        d.mode = MODES[mode]
        h = C.c_void_p()
        st = self.f["batch_create"](C.byref(d), arr, len(self.sims), C.byref(h))
        if st != abi.ST_OK:
            raise status_error("batch create", st)
        self._h = h
        self.mode = mode

    def set_mode(self, mode):
        st = self.f["batch_set_mode"](self._h, MODES[mode])
        if st != abi.ST_OK:
            raise status_error("batch set_mode", st)
        self.mode = mode

    def step(self, dt, opts):
        """opts[i]: tank i's options object (with its "cols" collider records, as SceneRunner builds them)."""
        packs = [make_opts(o, s.opt) for s, o in zip(self.sims, opts)]
        for s in self.sims:
            s.flushRun()
        ptrs = (C.POINTER(abi.StepOpts) * len(packs))(*[C.pointer(p[0]) for p in packs])
        st = self.f["batch_step"](self._h, float(dt), ptrs)
        if st != abi.ST_OK:
            raise status_error("batch step", st)
        del packs

    def set_sweeps(self, ctas_per_sm=8, wait_limit_us=1_000_000):
        """CTAs per SM of the pooled modes' sweeps, and the limit of each grid-barrier wait of the persistent one."""
        st = self.f["batch_set_sweeps"](self._h, int(ctas_per_sm), int(wait_limit_us))
        if st != abi.ST_OK:
            raise status_error("batch set_sweeps", st)

    def stream(self):
        return self.f["batch_stream"](self._h)

    def launches(self):
        return int(self.f["batch_launches"](self._h))

    def destroy(self):
        if getattr(self, "_h", None):
            self.f["batch_destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def lpt_partition(costs, parts):
    """Longest-processing-time split of tasks over parts: tasks by falling cost (index breaks ties), each to the part
    with the least load so far (lowest part index breaks ties). Returns one ascending list of task indices per part."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += costs[i]
    return [sorted(x) for x in out]


CANDIDATES = [(8, 4, 8), (4, 2, 4), (2, 2, 2), (1, 1, 1)]


def autotune(batch, sims, classes, run_step, timer, candidates=CANDIDATES, steps=3):
    """Coordinate search of the launch shape (st_flip_set_launch: heavy, light and pressure-sweep CTAs per SM) per
    class of tanks. classes: a list of lists of tank indices (e.g. small, medium, large). run_step() does one batch step;
    timer(fn) returns the device ms of fn(). Classes are tuned in the given order, each over the candidates with the
    others held; the step count per trial excludes one warm-up step that rebuilds the captured graphs. Results do not
    depend on the shape. Returns (choice per class, {trial: ms})."""
    choice = [candidates[0] for _ in classes]
    trials = {}

    def apply():
        for c, idx in zip(choice, classes):
            for i in idx:
                sims[i].set_launch(*c)

    for k, idx in enumerate(classes):
        if not idx:
            continue
        best = None
        for cand in candidates:
            choice[k] = cand
            apply()
            run_step()   # graphs are captured again for the new shape
            ms = timer(lambda: [run_step() for _ in range(steps)]) / steps
            trials[(k, cand)] = ms
            if best is None or ms < best[0]:
                best = (ms, cand)
        choice[k] = best[1]
    apply()
    return choice, trials


SCHEDULES = [("graph", 8), ("pooled", 8), ("pooled", 4), ("pooled", 16), ("persistent", 4), ("persistent", 2)]


def tune_schedule(batch, run_step, timer, schedules=SCHEDULES, steps=3):
    """The pressure-sweep schedule of a batch: each tank's own chained sweeps in its graph branch ("graph"), one pooled
    sweep launch per colour for all tanks ("pooled") or one persistent launch ("persistent"), at a number of CTAs per
    SM. Each is timed over `steps` batch steps after one that captures its graphs; the fastest is kept. Results do not
    depend on it. Returns (best (mode, ctas), {(mode, ctas): ms})."""
    trials = {}
    for mode, ctas in schedules:
        batch.set_mode(mode)
        batch.set_sweeps(ctas)
        run_step()
        trials[(mode, ctas)] = timer(lambda: [run_step() for _ in range(steps)]) / steps
    best = min(trials, key=lambda k: trials[k])
    batch.set_mode(best[0])
    batch.set_sweeps(best[1])
    return best, trials


def barrier_test(device=0, missing=1, limit_us=200_000):
    """The persistent sweep's bounded grid barrier with `missing` CTAs that never arrive: True when every wait ran out
    and the kernel returned with its error flag set (st_batch_barrier_test)."""
    out = C.c_uint32()
    st = funcs()["batch_barrier_test"](int(device), int(missing), int(limit_us), C.byref(out))
    if st != abi.ST_OK:
        raise status_error("batch barrier_test", st)
    return bool(out.value)


def wall_ms(fn, sync):
    t0 = time.perf_counter()
    fn()
    sync()
    return (time.perf_counter() - t0) * 1e3
