#!/usr/bin/env python
"""Benchmark of the B200 FLIP step: particle-steps/s on the full-feature 256^3 wave tank (one JSON line).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--workload wave_tank_256|wave_tank_256_band3|dam_break_64|pressure_512|batch_64|diff_128|pbf_dam]

One process per GPU (torchrun for N > 1, NCCL only for the barrier and the max/sum of the numbers). The FLIP step of
one tank does not shard, so N GPUs run N independent replica tanks (weak scaling) and value is the total over them.
Timing: W untimed steps, then K steps bracketed by a barrier and a device synchronise, CUDA events on the library's own
stream, the max over ranks. The working set (particles about 1.4 GB, grid about 0.6 GB) is larger than the 126 MB L2,
so no flush is needed between steps. --impl reference times the CPU restatement of the reference step (the oracle; the
reference's own step exists only as WGSL for a browser) on the host cores, on a bounded sample of the same scene.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# what limits each kernel instead of DRAM bandwidth, from ncu captures of the same kernels on the 128^3 wave tank
NCU_LIMITER = {"g2p": "instruction issue: 71% issue active at 24 warps per SM (80 registers), 998 instructions per particle",
               "p2g": "shared-memory atomics: L1 pipe 78% busy, 3.1 wavefronts per atomic (two thirds bank-conflict replays)"}
# dram__bytes_read.sum + dram__bytes_write.sum of one launch in a one-pass ncu capture of the 256^3 wave tank itself
# (the third step of `bench.py --steps 2 --warmup 1`, 37,847,049 live particles), scaled by the live particles
NCU_TRAFFIC = {"g2p": {"bytes": 1405361152 + 1227728640, "particles": 37847049},
               "p2g": {"bytes": 1697710848 + 1451466496, "particles": 37847049}}
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="wave_tank_256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=80)
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-extras", action="store_true", help="skip the pressure study and the 3-cell band run after the step")
    ap.add_argument("--tol", type=float, default=1e-6, help="pressure workloads: relative residual to reach")
    ap.add_argument("--omega", type=float, default=1.9, help="pressure workloads: SOR factor")
    ap.add_argument("--inner", type=int, default=100, help="pressure workloads: FP32 iterations per refinement")
    ap.add_argument("--ref-sweeps", type=int, default=1500, help="pressure workloads, reference arm: iterations the CPU time is scaled to")
    ap.add_argument("--no-autotune", action="store_true", help="batch workloads: default launch shapes")
    a = ap.parse_args()
    if a.workload.startswith("pressure_") and "--steps" not in sys.argv:
        a.steps, a.warmup = 5, 3
    if a.workload.startswith("batch_") and "--steps" not in sys.argv:
        a.steps = 100
    if a.workload.startswith("diff_") and "--steps" not in sys.argv:
        a.steps, a.warmup = 3, 1
    if a.workload.startswith("pbf_") and "--steps" not in sys.argv:
        a.steps, a.warmup = 30, 3
    return a


# ---------------------------------------------------------------- workloads
def workload(name):
    from splashtank_b200 import scenes
    if name.startswith("wave_tank"):
        # wave_tank_<n> (narrow band at full depth) or wave_tank_<n>_band<b> (a narrow band of b cells)
        parts = name.split("_")
        n = int(parts[2])
        band = float(parts[3][4:]) if len(parts) > 3 and parts[3].startswith("band") else 1e4
        return scenes.WaveTank(n, band=band)
    if name.startswith("dam_break"):
        n = int(name.rsplit("_", 1)[1])
        sc = scenes.dam_break(n)

        class Dam:
            pass
        w = Dam()
        w.__dict__.update(sc)
        w.states = lambda t: []
        w.spray_cap = 0
        w.opts = sc["opts"]

        def make(cls, **kw):
            s = cls(sc["d"], len(sc["pos"]), size=sc["size"], ratio=sc["ratio"], **kw)
            s.add_many(sc["pos"], sc["vel"])
            return s
        w.make = make
        return w
    raise SystemExit("unknown workload " + name)


def config_of(name, w, n_live):
    # particles (two 32-byte buffers) and the tile box's cells (about 94 bytes each) against the 126 MB L2
    n = getattr(w, "n", None) or int(round(1.0 / (2.0 * w.d)))
    ws = 64 * len(w.pos) + 94 * (math.ceil((n + 1) / 8.0) * 8) ** 3
    l2 = ("working set larger than L2 (126 MB): no flush" if ws > 126e6 else
          "working set (about %d MB) fits in L2: steps run back to back without a flush, each reading the state the one "
          "before left, as a running simulation does" % (ws // 1000000))
    cfg = {"workload": name, "particles": int(n_live), "dt": w.dt, "l2": l2, "parallelism": "replicas"}
    if name.startswith("wave_tank"):
        cfg.update(grid=[w.n] * 3, tile="8^3", sor_iters=w.opts["iters"],
                   narrow_band="full depth (band 1e4)" if w.band >= 1e4 else "%g cells" % w.band,
                   colliders="piston box 0.5 Hz amp 0.05 + sphere r 0.1 on a linear path over %d steps" % w.steps,
                   whitewater_cap=w.spray_cap,
                   pbf="not in this step (the 4-iteration PBF density stage is timed in the pbf4 and band3_pbf4 sub-objects)")
    return cfg


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, dev):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- algorithmic bytes per stage
def stage_bytes(stage, n, cells, fluid, iters):
    """Algorithmic HBM bytes of one launch of the stage's main kernel, and launches per step.
    n live particles, cells = 512 x tiles with storage, fluid = fluid cells. Per unit: a particle is 32 B (pos, vel),
    a cell's face data 24 B (three faces, two numbers each), cell count 4 B, pressure/rhs 4 B each, SOR info 2 B."""
    if stage == "g2p":        # read particle and write it back; read vn, vo of every face once, cell counts once
        return n * 64 + cells * (24 + 4), 1
    if stage == "p2g":        # read particle (and its id) from the old order, write it in sorted order; splat into face sums
        return n * 72 + cells * 24, 1
    if stage == "pressure":   # one colour sweep: own sorInfo, rhs, p read and p written; the other colour's p read once
        return fluid * (2 + 4 + 4 + 4) // 2 + fluid * 4 // 2, 2 * iters
    if stage == "blocks":     # read particle, write key and rank; sort scatter reads them, writes source index and id
        return n * (32 + 8 + 8 + 8), 1
    if stage == "norm_faces":  # read face sums, write vn and vo; read types, counts; write rhs and SOR info
        return cells * (24 + 24 + 4 + 4 + 4 + 2), 1
    if stage == "classify":
        return cells * (4 + 4 + 4 + 4), 1
    if stage == "project":    # vn read and written, p and types read, sums and other count buffer cleared
        return cells * (12 + 12 + 4 + 4 + 24 + 4), 1
    if stage == "narrow_band":
        return cells * (4 + 4 + 12) * 4, 4
    if stage == "reseed":
        return n * (32 + 4), 1
    if stage == "spray":
        return n * 32, 1
    return None, 1


def roofline(stage_ms, nsteps, n, cells, fluid, iters, peak, peak_src):
    dom = max((k for k in stage_ms if k != "total"), key=lambda k: stage_ms[k])
    b, launches = stage_bytes(dom, n, cells, fluid, iters)
    if not b or stage_ms[dom] <= 0:
        return None
    per_launch_ms = stage_ms[dom] / (nsteps * launches)
    achieved = b / (per_launch_ms * 1e-3) / 1e9
    # DRAM bytes of one launch from an ncu capture of the same tank, scaled by the live particles of this run
    ent = NCU_TRAFFIC.get(dom)
    traffic = int(ent["bytes"] * n / ent["particles"]) if ent else None
    return {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src, "traffic": traffic,
            "algorithmic_bytes_per_launch": int(b), "launch_ms": round(per_launch_ms, 5),
            "stage_share": round(stage_ms[dom] / stage_ms["total"], 4), "limiter": NCU_LIMITER.get(dom)}


def step_bytes_model(n, cells, fluid, iters, nb_on, ww_slots, sort_every=16):
    """Algorithmic HBM bytes of one whole step by the per-unit model of the reference's state layout: particles 112 B
    (tile marking reads pos 16, P2G reads pos and vel 32, G2P reads 32 and writes 32) plus the sort's copies (pos, vel
    and id in and out, 72 B) every sort_every steps (the reference sorts every 16th step; this library's sort is part of
    P2G's gather every step and is not counted again); grid 168 B per cell with storage (P2G sums and count 28, classify
    8, normFaces 48, divergence 24, project 32, G2P face reads 24, clear 4); the red-black SOR 16 B per fluid cell and
    iteration; the narrow band 56 B per cell (four 8-byte passes and the kept velocity); whitewater 32 B per particle
    (the emission read) and 64 B per handed-out point (its sample and step)."""
    b = 112 * n + 72 * n / sort_every + 168 * cells + 16 * fluid * iters
    if nb_on:
        b += 56 * cells
    if ww_slots is not None:
        b += 32 * n + 64 * ww_slots
    return int(b)


def step_roofline(ms_per_step, n, cells, fluid, iters, nb_on, ww_slots, stage_ms, nrec, peak, peak_src):
    """The whole step against the HBM roofline: algorithmic bytes of a step (step_bytes_model) over the device time of
    a step, and beside it the sum of the per-kernel figures of stage_bytes over the stages that ran."""
    b = step_bytes_model(n, cells, fluid, iters, nb_on, ww_slots)
    ach = b / (ms_per_step * 1e-3) / 1e9
    kb = 0
    for k in stage_ms:
        if k == "total" or stage_ms[k] <= 0:
            continue
        x, launches = stage_bytes(k, n, cells, fluid, iters)
        kb += (x or 0) * launches
    return {"step_bytes": b, "step_ms": round(ms_per_step, 4), "step_achieved": round(ach, 1), "step_frac": round(ach / peak, 4),
            "kernel_bytes": int(kb), "kernel_frac": round(kb / (ms_per_step * 1e-3) / 1e9 / peak, 4),
            "target_ms_at_60pct": round(b / (0.6 * peak * 1e9) * 1e3, 4), "peak": peak, "peak_source": peak_src,
            "model": "112 B/particle + 72 B/particle sort copies + 168 B/cell + 16 B/fluid cell/iteration + 56 B/cell narrow band "
                     "+ 32 B/particle + 64 B/point whitewater"}


def measured_peak():
    try:
        p = json.load(open(PEAKS))
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM, "fallback 6.65 TB/s"


# ---------------------------------------------------------------- CPU baseline (oracle)
def cpu_sample(name, w=None, budget_s=20.0, threads=None, warm=1):
    """Time the CPU restatement (all host threads) on a bounded sample of the same workload: `warm` untimed steps, then
    steps until budget_s has passed (at least one). w: the workload object already built for the GPU run, if any."""
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.scene import SceneRunner
    w = w or workload(name)
    th = threads or os.cpu_count() or 1
    sim = w.make(OracleFlipSim, threads=th)
    run = SceneRunner(sim)
    t = 0.0
    for _ in range(warm):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    k, t0 = 0, time.perf_counter()
    while True:
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
        k += 1
        el = time.perf_counter() - t0
        if el > budget_s:
            break
    live = sim.readStats()["live"]
    sim.destroy()
    return {"value": live * k / el, "unit": "particle-steps/s", "cores": th, "kind": "port",
            "sample": "%s (%d live particles): %d steps after %d untimed, oracle with %d OpenMP threads (%.1f s)" % (name, live, k, warm, th, el)}, el


def run_reference(a):
    """The reference arm: the reference's FLIP step exists only as WGSL for a browser (no graphics stack here), so its
    CPU restatement (the oracle, all host threads) steps the same workload; each timed step is a whole step of that
    workload, and the timed steps are bounded (at most 10 after at most 1 untimed) so the arm ends within minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.scene import SceneRunner
    w = workload(a.workload)
    th = os.cpu_count() or 1
    sim = w.make(OracleFlipSim, threads=th)
    run = SceneRunner(sim)
    warm, steps = min(a.warmup, 1), max(1, min(a.steps, 10))
    t = 0.0
    for _ in range(warm):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    t0 = time.perf_counter()
    for _ in range(steps):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    el = time.perf_counter() - t0
    live = sim.readStats()["live"]
    v = live * steps / el
    sample = ("%s (%d live particles): %d steps after %d untimed, the oracle with %d OpenMP threads; the reference's FLIP step runs "
              "only as WGSL in a browser (no graphics stack here), so its CPU restatement stands in" % (a.workload, live, steps, warm, th))
    line = {"metric": "particle-steps/s", "value": v, "unit": "particle-steps/s", "impl": "reference", "n_gpus": a.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": el * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": config_of(a.workload, w, live),
            "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": th, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- pressure solve precision study
def pressure_scene(name):
    from splashtank_b200 import scenes
    n = int(name.rsplit("_", 1)[1])
    ty, rhs = scenes.splash_blobs(n)
    return n, ty, rhs


def pressure_config(name, n, ty, nt, a):
    return {"workload": name, "grid": [n] * 3, "tile": "8^3", "active_tiles": nt, "active_tile_frac": round(nt / (n // 8) ** 3, 4),
            "fluid_cells": int((ty == 1).sum()), "tol": a.tol, "omega": a.omega, "inner_sweeps": a.inner,
            "scene": "seeded Gaussian blobs above 0.5 (120 blobs, sigma 0.025-0.07 of the box), solid walls; rhs = divergence of a "
                     "seeded uniform(-1,1) face field", "l2": "working set (FP32 p, rhs about 250 MB at 512^3) larger than L2: no flush",
            "parallelism": "replicas"}


def run_pressure(a):
    """ms per pressure solve to rel residual tol: FP32 SOR inside FP64 refinement (the value), plain FP32 SOR and FP64 SOR
    beside it, each solution's error against an FP64 SOR solve to 1e-11 (the FP64 operator and its CG solution are checked
    against the oracle in the tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    from splashtank_b200.poisson import REFINE, SOR32, SOR64, PoissonSolver
    n, ty, rhs = pressure_scene(a.workload)
    s = PoissonSolver((n, n, n), device=local)
    t0 = time.perf_counter()
    s.set(ty, rhs)
    nt, nf = s.stats()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # every solve checks its residual on the same schedule: blocks sized from the last block's reduction per iteration
    # (at most a.inner iterations), so that no solver runs up to a block past the tolerance
    ro = dict(tol=a.tol, omega=a.omega, inner_sweeps=a.inner, max_sweeps=200000, predict=True)
    for _ in range(a.warmup):
        s.solve(REFINE, **ro)
    clocks = Clocks(local)
    barrier()
    res = [s.solve(REFINE, **ro) for _ in range(a.steps)]
    barrier()
    clk = clocks.stop()
    ms = sum(r["ms"] for r in res)
    if dist:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_per = ms / a.steps
    r_ref = res[-1]
    x_ref32 = s.read()
    # plain FP32 SOR to the same tolerance (residual checked as often as the refinement checks it), then FP64 SOR
    r32 = s.solve(SOR32, tol=a.tol, omega=a.omega, check_every=a.inner, max_sweeps=max(4 * r_ref["sweeps"], 2000), predict=True)
    x32 = s.read()
    r64 = s.solve(SOR64, tol=a.tol, omega=a.omega, check_every=a.inner, max_sweeps=max(4 * r_ref["sweeps"], 2000), predict=True)
    x64 = s.read()
    # the same two with fixed blocks of a.inner iterations between checks
    fixed = {k: s.solve(m, tol=a.tol, omega=a.omega, inner_sweeps=a.inner, check_every=a.inner, max_sweeps=max(4 * r_ref["sweeps"], 2000))
             for k, m in (("refine", REFINE), ("fp32_sor", SOR32))}
    # a tighter target: FP32 SOR stops improving at its rounding floor, the refinement keeps going at FP32 sweep cost
    t9 = 1e-9
    r9 = s.solve(REFINE, tol=t9, omega=a.omega, inner_sweeps=a.inner, max_sweeps=20000, predict=True)
    r9_32 = s.solve(SOR32, tol=t9, omega=a.omega, check_every=a.inner, max_sweeps=max(2 * r9["sweeps"], 2000), predict=True)
    r9_64 = s.solve(SOR64, tol=t9, omega=a.omega, check_every=a.inner, max_sweeps=max(2 * r9["sweeps"], 2000), predict=True)
    rgold = s.solve(SOR64, tol=1e-11, omega=a.omega, check_every=50, max_sweeps=400000)
    gold = s.read()
    gn, gmax = float(np.linalg.norm(gold)), float(np.abs(gold).max())

    def err(x):
        d = x - gold
        return {"rel_l2": float(np.linalg.norm(d)) / gn, "max_abs_over_max": float(np.abs(d).max()) / gmax}
    # roofline of the FP32 sweep kernel (one colour per launch): per launch every cell of the active tiles reads its 2-byte
    # info word in its own colour half, and every fluid cell of the colour reads rhs and p, writes p, and one fluid cell
    # of the other colour is read (4 B): cells/2 * 2 + fluid/2 * 16 bytes
    it = 200
    sms = s.sweeps32(a.omega, it)
    per_launch = sms / (2 * it)
    b = nt * 512 + nf * 8
    peak, src = measured_peak()
    achieved = b / (per_launch * 1e-3) / 1e9
    rl = {"kernel": "k_ps_sor32", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
          "peak_source": src, "traffic": None, "algorithmic_bytes_per_launch": int(b), "launch_ms": round(per_launch, 5)}
    # end to end through the C ABI with host buffers: upload (types, rhs), solve, read back
    e0 = time.perf_counter()
    s.set(ty, rhs)
    re = s.solve(REFINE, **ro)
    s.read()
    e_ms = (time.perf_counter() - e0) * 1e3
    if rank == 0:
        line = {"metric": "pressure ms/solve to 1e-6 rel residual (FP32 SOR in FP64 refinement)", "value": ms_per, "unit": "ms",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 sweeps, f64 residual/correction", "data": "synthetic (seeded)",
                "config": pressure_config(a.workload, n, ty, nt, a), "gpu_launches": int(r_ref["sweeps"] * 2 + r_ref["refinements"] * 4 + 2),
                "refine": {"ms": ms_per, "sweeps": r_ref["sweeps"], "refinements": r_ref["refinements"], "rel_residual": r_ref["rel_residual"],
                           "error_vs_fp64": err(x_ref32)},
                "fp32_sor": {"ms": r32["ms"], "sweeps": r32["sweeps"], "rel_residual": r32["rel_residual"], "converged": r32["converged"],
                             "error_vs_fp64": err(x32)},
                "fp64_sor": {"ms": r64["ms"], "sweeps": r64["sweeps"], "rel_residual": r64["rel_residual"], "converged": r64["converged"],
                             "error_vs_fp64": err(x64)},
                "fp64_reference": {"method": "FP64 SOR to 1e-11", "sweeps": rgold["sweeps"], "rel_residual": rgold["rel_residual"], "ms": rgold["ms"]},
                "tol_1e-9": {k: {"ms": r["ms"], "sweeps": r["sweeps"], "rel_residual": r["rel_residual"], "converged": r["converged"]}
                             for k, r in (("refine", r9), ("fp32_sor", r9_32), ("fp64_sor", r9_64))},
                "schedule": "checks after blocks sized from the last block's reduction per iteration (8 to %d iterations)" % a.inner,
                "fixed_blocks": {k: {"ms": r["ms"], "sweeps": r["sweeps"], "refinements": r["refinements"], "rel_residual": r["rel_residual"]}
                                 for k, r in fixed.items()},
                "clocks": clk, "roofline": rl,
                "e2e": {"value": e_ms, "unit": "ms", "h2d_bytes_per_step": int(ty.nbytes + rhs.nbytes), "d2h_bytes_per_step": int(gold.nbytes),
                        "note": "wall clock of set (host builds the tile index) + solve + read through the C ABI"}}
        if world == 1 and not a.no_cpu_baseline:
            line["cpu_baseline"] = pressure_cpu(ty, rhs, n, a, r_ref["sweeps"])
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def pressure_cpu(ty, rhs, n, a, sweeps, budget_sweeps=6):
    """The oracle's FP32 SOR sweeps (all host threads) on the same system, a few sweeps timed and scaled to the sweep
    count the refined solve needs."""
    from oracle.oracle import OraclePoisson
    th = os.cpu_count() or 1
    o = OraclePoisson((n, n, n), threads=th)
    o.set(ty, rhs)
    o.sweeps32(a.omega, 1)
    t0 = time.perf_counter()
    o.sweeps32(a.omega, budget_sweeps)
    el = time.perf_counter() - t0
    v = el * 1e3 / budget_sweeps * sweeps
    return {"value": v, "unit": "ms", "cores": th, "kind": "port",
            "sample": "%d FP32 SOR iterations of the oracle on the %d^3 system timed (%.1f s), scaled to the %d iterations of the "
                      "refined solve" % (budget_sweeps, n, el, sweeps)}


def run_pressure_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n, ty, rhs = pressure_scene(a.workload)
    cb = pressure_cpu(ty, rhs, n, a, a.ref_sweeps)
    line = {"metric": "pressure ms/solve to 1e-6 rel residual (FP32 SOR in FP64 refinement)", "value": cb["value"], "unit": "ms",
            "impl": "reference", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": cb["value"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": a.workload, "grid": [n] * 3, "tol": a.tol, "omega": a.omega},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pressure_summary(local, tol=1e-6, omega=1.9, inner=100, repeats=3, n=512):
    """The metric's pressure half, run after the FLIP step's timed region: ms per solve of the 512^3 splash system to
    `tol` relative residual, FP32 SOR inside FP64 refinement against plain FP32 SOR (the median of `repeats` solves each,
    the same predicted check schedule for both), each solution's error against an FP64 SOR solve to 1e-11, and the same
    comparison at 1e-9, where FP32 SOR stalls at its rounding floor."""
    from splashtank_b200.poisson import REFINE, SOR32, SOR64, PoissonSolver
    ty, rhs = pressure_scene("pressure_%d" % n)[1:]
    s = PoissonSolver((n, n, n), device=local)
    s.set(ty, rhs)
    nt, nf = s.stats()
    ro = dict(tol=tol, omega=omega, inner_sweeps=inner, max_sweeps=200000, predict=True)
    s.solve(REFINE, **ro)   # warm-up
    out = {}
    for key, mode in (("refine", REFINE), ("fp32_sor", SOR32)):
        runs = []
        for _ in range(repeats):
            kw = dict(ro) if mode == REFINE else dict(tol=tol, omega=omega, check_every=inner, max_sweeps=20000, predict=True)
            runs.append(s.solve(mode, **kw))
        runs.sort(key=lambda r: r["ms"])
        r = runs[len(runs) // 2]
        out[key] = {"ms": r["ms"], "ms_runs": [round(x["ms"], 3) for x in runs], "sweeps": r["sweeps"], "refinements": r["refinements"],
                    "rel_residual": r["rel_residual"], "converged": r["converged"], "x": s.read()}
    r9 = {"refine": s.solve(REFINE, tol=1e-9, omega=omega, inner_sweeps=inner, max_sweeps=20000, predict=True)}
    r9["fp32_sor"] = s.solve(SOR32, tol=1e-9, omega=omega, check_every=inner, max_sweeps=2 * r9["refine"]["sweeps"], predict=True)
    rgold = s.solve(SOR64, tol=1e-11, omega=omega, check_every=50, max_sweeps=400000)
    gold = s.read()
    s.destroy()
    gn, gmax = float(np.linalg.norm(gold)), float(np.abs(gold).max())
    for k in out:
        d = out[k].pop("x") - gold
        out[k]["error_vs_fp64"] = {"rel_l2": float(np.linalg.norm(d)) / gn, "max_abs_over_max": float(np.abs(d).max()) / gmax}
    out.update(workload="pressure_%d" % n, tol=tol, omega=omega, active_tiles=nt, fluid_cells=nf,
               refine_vs_fp32_speedup=round(out["fp32_sor"]["ms"] / out["refine"]["ms"], 4),
               fp64_reference={"method": "FP64 SOR to 1e-11", "sweeps": rgold["sweeps"], "rel_residual": rgold["rel_residual"]},
               tol_1e9={k: {"ms": r["ms"], "sweeps": r["sweeps"], "rel_residual": r["rel_residual"], "converged": r["converged"]}
                        for k, r in r9.items()},
               scene="seeded Gaussian blobs (120, sigma 0.025-0.07 of the box) above 0.5 inside solid walls; rhs = divergence of a "
                     "seeded uniform(-1,1) face field", unit="ms per solve, CUDA events on the solver's stream")
    return out


def band_summary(local, name="wave_tank_256_band3", warm=8, steps=20):
    """The wave tank with the reference's narrow band of 3 cells (particles only in the band under the surface after
    the first steps trim the deep water), device-timed like the headline run."""
    import torch
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = workload(name)
    sim = w.make(FlipSim, device=local)
    run = SceneRunner(sim)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    t = 0.0
    for _ in range(warm):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    st = sim.readStats()
    sim.destroy()
    return {"workload": name, "value": st["live"] * steps / (ms * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms / steps,
            "live_particles": st["live"], "seeded_particles": len(w.pos), "tiles_with_storage": st["sc"], "fluid_cells": st["fluid"],
            "steps": steps, "warmup": warm, "narrow_band": "3 cells (deep calm particles trimmed, thin band cells refilled)"}


def pbf4_summary(local, name="wave_tank_256", iters=4, warm=3, steps=8):
    """The headline tank with the PBF density stage of 4 iterations at the end of every step (st_step_opts.pbf_iters):
    the configuration's "PBF density constraints with 4 iterations", device-timed like the headline run."""
    import torch
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = workload(name)
    w.opts = dict(w.opts, pbf=iters)
    sim = w.make(FlipSim, device=local)
    run = SceneRunner(sim)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    t = 0.0
    sim.set_timing(True)
    for _ in range(warm):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    torch.cuda.synchronize()
    sim.read_timing()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    stages, nrec = sim.read_timing()
    st = sim.readStats()
    sim.destroy()
    return {"workload": name, "pbf": "%d iterations (GpuSim's density constraint, kernel radius 2.2 d)" % iters,
            "value": st["live"] * steps / (ms * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms / steps,
            "pbf_stage_ms": stages["pbf"] / max(nrec, 1), "flip_stages_ms": (stages["total"] - stages["pbf"]) / max(nrec, 1),
            "particles": st["live"], "steps": steps, "warmup": warm}


def batch_summary(local, count=64, warm=2, steps=10):
    """Config 5 after the headline's timed region: the 64 uneven tanks stepped together with the sweep schedule picked
    by the autotuner (graph branches, or the shared pool swept by one launch per colour or one persistent launch),
    against the same step graphs as parallel branches and launched one after another; device-timed, 1 GPU."""
    import torch
    from splashtank_b200 import scenes
    from splashtank_b200.batch import TankBatch, tune_schedule
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    spec = scenes.BatchTanks(count=count)
    made = [spec.make(k, FlipSim, device=local) for k in range(count)]
    sims = [m[0] for m in made]
    runners = [SceneRunner(s) for s in sims]
    batch = TankBatch(sims, "graph")
    stream = torch.cuda.ExternalStream(batch.stream(), device=local)

    def step():
        batch.step(spec.dt, [spec.step_opts(k, s, r) for k, s, r in zip(range(count), sims, runners)])

    def timer(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(warm):
        step()
    sched, trials = tune_schedule(batch, step, timer)
    out = {}
    for name, mode in (("tuned", sched[0]), ("graph_branches", "graph"), ("sequential", "sequential")):
        batch.set_mode(mode)
        for _ in range(warm):
            step()
        ms = timer(lambda: [step() for _ in range(steps)]) / steps
        out[name] = ms
    live = sum(s.readStats()["live"] for s in sims)
    batch.destroy()
    for s in sims:
        s.destroy()
    return {"workload": "batch_%d" % count, "tanks": count, "particles": int(live), "unit": "particle-steps/s",
            "value": live / (out["tuned"] * 1e-3), "ms_per_step": out["tuned"],
            "sweep_schedule": {"mode": sched[0], "ctas_per_sm": sched[1]},
            "schedule_trials_ms": {"%s:%d" % k: round(v, 3) for k, v in trials.items()},
            "graph_branches_ms_per_step": out["graph_branches"], "sequential_ms_per_step": out["sequential"],
            "speedup_vs_sequential": round(out["sequential"] / out["tuned"], 3), "steps": steps, "warmup": warm,
            "launch_shape": "default (the full autotune of launch shapes runs in --workload batch_64)"}


def diff_summary(local, n=128):
    """Config 4 after the headline's timed region: one FP32 gradient of the 32-step rollout (forward with checkpoints,
    recompute, adjoint) and the forward alone, with the distance-grid box collider, and the FP32 gradient against the
    FP64 one."""
    import torch
    from splashtank_b200 import scenes
    d = scenes.DiffDam(n=n)
    p0 = d.params
    s32 = d.make(collider="grid", device=local)
    stream = torch.cuda.ExternalStream(s32.stream(), device=local)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    s32.forward(p0)
    s32.backward()
    ms_grad = timed(lambda: (s32.forward(p0), s32.backward()))
    ms_fwd = timed(lambda: s32.forward(p0))
    s32.forward(p0)
    g32 = s32.backward()
    s32.destroy()
    s64 = d.make(fp64=True, collider="grid", device=local)
    s64.forward(p0)
    g64 = s64.backward()
    s64.destroy()
    ps = d.pos.shape[0] * d.steps
    return {"workload": "diff_%d" % n, "particles": int(d.pos.shape[0]), "rollout_steps": d.steps, "checkpoint_every": d.ckpt,
            "collider": "the box's distance grid (sdfEval's trilinear gradient and Hessian in the adjoint)",
            "gradient_ms": ms_grad, "forward_ms": ms_fwd, "value": ps / (ms_grad * 1e-3), "unit": "gradient particle-steps/s",
            "f32_vs_f64_adjoint_rel_l2": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))}


# ---------------------------------------------------------------- the PBF engine (GpuSim)
def pbf_scene(name):
    """pbf_dam: GpuSim's dam break in the app's default box (3 x 2.6 x 3): water where x < 0 and y < 1.3 on FluidSim's
    lattice at spacing d = 0.0125 with its jitter (seeded): 2,995,200 particles; a sphere collider of radius 0.3 as a
    distance grid; gravity 9.81, XSPH viscosity 0.02, 4 solver iterations, dt 1/120."""
    from splashtank_b200.scene import sphere_sdf
    d = 0.0125
    rng = np.random.default_rng(9)
    j = 0.01 * d / 0.12
    ys, xs, zs = np.arange(d / 2, 1.3, d), np.arange(-1.5 + d / 2, 0.0, d), np.arange(-1.5 + d / 2, 1.5, d)
    Y, X, Z = np.meshgrid(ys, xs, zs, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    pos = (pos + (rng.random(pos.shape) - 0.5) * j).astype(np.float32)
    sph = sphere_sdf(0.3, 0.02, sid=1)
    opts = dict(g=9.81, iters=4, visc=0.02, cols=[dict(sdf=sph, x=0.6, y=0.3, z=0.0)])
    return dict(d=d, pos=pos, opts=opts, dt=1.0 / 120.0)


def pbf_bytes(n, iters):
    """Algorithmic HBM bytes of one PBF step by the per-unit model (8 + 2 iters) x 32 B per particle: the particle state
    read and written by predict, finalize and viscosity, and twice per iteration the sorted positions and multipliers;
    neighbour reads are served from the caches and not counted."""
    return (8 + 2 * iters) * 32 * n


def run_pbf(a):
    """particle-steps/s of the PBF engine (st_pbf_step, GpuSim's semantics) on pbf_dam; the GpuSim restatement (the
    oracle, all host threads) on a bounded sample of steps of the same scene beside it."""
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    from splashtank_b200.pbf import PbfSim
    sc = pbf_scene(a.workload)
    n = len(sc["pos"])
    s = PbfSim(sc["d"], n, device=local)
    s.add_many(sc["pos"])
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    for _ in range(a.warmup):
        s.step(sc["dt"], sc["opts"])
    torch.cuda.synchronize()
    clocks = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        s.step(sc["dt"], sc["opts"])
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    # end to end: parameters and collider records up, every particle (position and velocity) back each step
    pin = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True).numpy()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, a.steps // 2)
    import ctypes as C
    from splashtank_b200 import abi
    pp = pin[:n * 16].view(np.float32)
    vv = pin[n * 16:].view(np.float32)
    got = C.c_uint32()
    f0.record(stream)
    for _ in range(e2e_steps):
        s.step(sc["dt"], sc["opts"])
        s.f["pbf_read"](s._h, pp.ctypes.data_as(abi.f32p), vv.ctypes.data_as(abi.f32p), n, C.byref(got))
    f1.record(stream)
    f1.synchronize()
    ems = f0.elapsed_time(f1)
    s.destroy()
    if rank == 0:
        peak, src = measured_peak()
        per = ms / a.steps
        b = pbf_bytes(n, sc["opts"]["iters"])
        line = {"metric": "particle-steps/s", "value": n * a.steps / (ms * 1e-3), "unit": "particle-steps/s", "n_gpus": 1, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": per, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded lattice jitter)",
                "config": {"workload": a.workload, "particles": n, "d": sc["d"], "iters": sc["opts"]["iters"], "visc": sc["opts"]["visc"],
                           "dt": sc["dt"], "colliders": "sphere r 0.3 (distance grid)", "box": [3.0, 2.6, 3.0],
                           "l2": "working set larger than L2: no flush", "parallelism": "replicas"},
                "gpu_launches": int(a.steps * (6 + 2 * sc["opts"]["iters"] + 2)), "clocks": clk,
                "roofline": {"kernel": "whole PBF step", "bound": "hbm", "achieved": round(b / (per * 1e-3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(b / (per * 1e-3) / 1e9 / peak, 4), "peak_source": src, "traffic": None,
                             "algorithmic_bytes_per_launch": int(b), "launch_ms": round(per, 4),
                             "limiter": "the 27-cell neighbour loops (about 290 candidates per particle per pass): issue and L1 latency"},
                "e2e": {"value": n * e2e_steps / (ems * 1e-3), "unit": "particle-steps/s", "h2d_bytes_per_step": 64 + 128,
                        "d2h_bytes_per_step": n * 32, "steps": e2e_steps, "readback": "every particle's position and velocity each step"}}
        if not a.no_cpu_baseline:
            line["cpu_baseline"] = pbf_cpu(sc)
        print(json.dumps(line), flush=True)


def pbf_cpu(sc, budget_s=20.0, steps=None):
    """The GpuSim restatement (all host threads) on the same scene: steps until budget_s has passed (at least one)."""
    from oracle.oracle import OraclePbfSim
    th = os.cpu_count() or 1
    n = len(sc["pos"])
    o = OraclePbfSim(sc["d"], n, threads=th)
    o.add_many(sc["pos"])
    o.step(sc["dt"], sc["opts"])
    k, t0 = 0, time.perf_counter()
    while True:
        o.step(sc["dt"], sc["opts"])
        k += 1
        el = time.perf_counter() - t0
        if (steps and k >= steps) or (not steps and el > budget_s):
            break
    o.destroy()
    return {"value": n * k / el, "unit": "particle-steps/s", "cores": th, "kind": "port",
            "sample": "pbf_dam (%d particles): %d steps after 1 untimed, the GpuSim restatement with %d OpenMP threads (%.1f s)" % (n, k, th, el)}


def run_pbf_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc = pbf_scene(a.workload)
    cb = pbf_cpu(sc, steps=max(1, min(a.steps, 10)))
    line = {"metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s", "impl": "reference", "n_gpus": a.gpus,
            "steps": max(1, min(a.steps, 10)), "warmup": 1, "ms_per_step": len(sc["pos"]) / cb["value"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice jitter)",
            "config": {"workload": a.workload, "particles": len(sc["pos"])}, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- many tanks per step
def batch_bytes(stats, iters):
    """Algorithmic HBM bytes of one step of every tank (the stage_bytes figures of the main stages, summed)."""
    tot = 0
    for live, tiles, fluid in stats:
        cells = tiles * 512
        for st in ("blocks", "p2g", "norm_faces", "classify", "project", "g2p"):
            b, _ = stage_bytes(st, live, cells, fluid, iters)
            tot += b
        b, launches = stage_bytes("pressure", live, cells, fluid, iters)
        tot += b * launches
    return tot


def run_batch(a):
    """64 tanks of uneven size stepped together: value = particle-steps/s over all tanks with the step graphs of all of
    a rank's tanks in one graph launch and launch shapes from the autotuner; the same tanks launched one after another
    are timed beside it. Ranks take disjoint sets of tanks (LPT on cells + particles); no collective in the step."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    from splashtank_b200 import scenes
    from splashtank_b200.batch import TankBatch, autotune, lpt_partition, tune_schedule
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    count = int(a.workload.rsplit("_", 1)[1])
    spec = scenes.BatchTanks(count=count)
    mine = lpt_partition([spec.cost(k) for k in range(count)], world)[rank]
    made = [spec.make(k, FlipSim, device=local) for k in mine]
    sims = [m[0] for m in made]
    runners = [SceneRunner(s) for s in sims]
    batch = TankBatch(sims, "graph")
    stream = torch.cuda.ExternalStream(batch.stream(), device=local)

    def step():
        batch.step(spec.dt, [spec.step_opts(k, s, r) for k, s, r in zip(mine, sims, runners)])

    def timer(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t)
        return float(t.item())

    for _ in range(2):
        step()
    # autotune the launch shape per size class (thirds of this rank's tanks by cells)
    order = sorted(range(len(mine)), key=lambda i: spec.cost(mine[i]))
    third = max(1, len(order) // 3)
    classes = [order[:third], order[third:2 * third], order[2 * third:]]
    choice, trials = autotune(batch, sims, classes, step, timer) if not a.no_autotune else ([(8, 4, 8)] * 3, {})
    # the pressure-sweep schedule: per-tank chains in graph branches, the shared pool swept by one launch per colour, or
    # one persistent cooperative launch
    sched, sched_ms = tune_schedule(batch, step, timer) if not a.no_autotune else (("graph", 8), {})
    for _ in range(a.warmup):
        step()
    barrier()
    l0 = batch.launches()
    clocks = Clocks(local)
    barrier()
    ms = timer(lambda: [step() for _ in range(a.steps)])
    barrier()
    clk = clocks.stop()
    launches = batch.launches() - l0
    stats = [s.readStats() for s in sims]
    live = sum(st["live"] for st in stats)
    ms_max = max_over_ranks(ms)
    live_all = sum_over_ranks(live)
    value = live_all * a.steps / (ms_max * 1e-3)
    # the same tanks, one step graph after another on one stream
    batch.set_mode("sequential")
    for _ in range(2):
        step()
    barrier()
    ms_seq = max_over_ranks(timer(lambda: [step() for _ in range(a.steps)]))
    # every tank's step graph as a parallel branch of one launch (the per-tank sweep chains), for comparison
    batch.set_mode("graph")
    for _ in range(2):
        step()
    barrier()
    ms_branch = max_over_ranks(timer(lambda: [step() for _ in range(a.steps)]))
    batch.set_mode(sched[0])
    # end to end: every step the options and collider records go up and every tank's counters come back
    barrier()
    e_steps = max(1, a.e2e_steps // 4)
    ems = max_over_ranks(timer(lambda: [(step(), [s.readStats() for s in sims]) for _ in range(e_steps)]))
    if rank == 0:
        peak, src = measured_peak()
        iters = spec.opts["iters"]
        b = batch_bytes([(st["live"], st["sc"], st["fluid"]) for st in stats], iters)
        per_step_ms = ms / a.steps
        achieved = b / (per_step_ms * 1e-3) / 1e9
        ntanks = len(mine)
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded tanks, 8 particles per cell)",
                "config": {"workload": a.workload, "tanks": count, "tanks_rank0": ntanks, "particles": int(live_all),
                           "edges": "uniform from %s per axis, cell 1/64" % (scenes.TANK_EDGES,), "fill": "20-60%",
                           "collider": "one static SDF sphere per tank", "sor_iters": iters, "dt": spec.dt,
                           "mode": {"graph": "one graph launch per step (tank step graphs as parallel branches)",
                                    "pooled": "one graph per step: tank branches, then every tank's fluid tiles in one shared pool swept by "
                                              "one launch per colour, then tank branches",
                                    "persistent": "tank branches, one persistent cooperative launch for all sweeps of all tanks (bounded "
                                                  "grid-barrier waits), tank branches"}[sched[0]],
                           "sweep_schedule": {"mode": sched[0], "ctas_per_sm": sched[1]},
                           "launch_shape_per_class": choice, "parallelism": "tanks split over ranks (LPT)",
                           "l2": "working set larger than L2: no flush"},
                "gpu_launches": int(launches),
                "sequential": {"ms_per_step": ms_seq / a.steps, "value": live_all * a.steps / (ms_seq * 1e-3),
                               "mode": "the same step graphs launched one after another on one stream"},
                "graph_branches": {"ms_per_step": ms_branch / a.steps, "value": live_all * a.steps / (ms_branch * 1e-3),
                                   "mode": "every tank's step graph as a parallel branch of one launch"},
                "schedule_ms": {"%s:%d" % k: round(v, 3) for k, v in sched_ms.items()},
                "autotune_ms": {"%d:%s" % (k, "x".join(map(str, c))): round(v, 3) for (k, c), v in trials.items()},
                "clocks": clk,
                "roofline": {"kernel": "whole batch step (all kernels of all tanks)", "bound": "hbm", "achieved": round(achieved, 1),
                             "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": src, "traffic": None,
                             "algorithmic_bytes_per_launch": int(b), "launch_ms": round(per_step_ms, 4)},
                "e2e": {"value": live_all * e_steps / (ems * 1e-3), "unit": "particle-steps/s",
                        "h2d_bytes_per_step": int(ntanks * (496 + 128)), "d2h_bytes_per_step": int(ntanks * 64), "steps": e_steps,
                        "readback": "every tank's counters every step"}}
        if world == 1 and not a.no_cpu_baseline:
            line["cpu_baseline"] = batch_cpu(spec)
        print(json.dumps(line), flush=True)
    batch.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def batch_cpu(spec, budget_s=15.0):
    """The oracle (all host threads) stepping the smallest tanks of the set one after another, a bounded sample."""
    from oracle.oracle import OracleFlipSim
    from splashtank_b200.scene import SceneRunner
    th = os.cpu_count() or 1
    order = sorted(range(len(spec.tanks)), key=lambda k: spec.cost(k))[:4]
    sims = [spec.make(k, OracleFlipSim, threads=th)[0] for k in order]
    runners = [SceneRunner(s) for s in sims]
    n, steps, t0 = 0, 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        for k, s, r in zip(order, sims, runners):
            s.step(spec.dt, spec.step_opts(k, s, r))
        steps += 1
    el = time.perf_counter() - t0
    n = sum(s.readStats()["live"] for s in sims)
    return {"value": n * steps / el, "unit": "particle-steps/s", "cores": th, "kind": "port",
            "sample": "the 4 smallest tanks (%d particles), %d steps each, oracle with %d OpenMP threads" % (n, steps, th)}


def run_batch_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from splashtank_b200 import scenes
    spec = scenes.BatchTanks(count=int(a.workload.rsplit("_", 1)[1]))
    cb = batch_cpu(spec, budget_s=min(60.0, 5.0 * max(1, a.steps)))
    line = {"metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s", "impl": "reference", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded tanks)", "config": {"workload": a.workload}, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- differentiable rollout
def run_diff(a):
    """Gradient of the 32-step differentiable rollout (forward with checkpoints, recompute, adjoint) in FP32: value =
    particle-steps/s of the whole gradient evaluation; beside it the forward alone, and the gradient's error against
    the FP64 adjoint and against FP64 central differences (eps 1e-3) on six parameters."""
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    from splashtank_b200 import scenes
    n = int(a.workload.rsplit("_", 1)[1])
    d = scenes.DiffDam(n=n)
    p0 = d.params
    s32 = d.make(device=local)
    stream = torch.cuda.ExternalStream(s32.stream(), device=local)

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    for _ in range(a.warmup):
        s32.forward(p0)
        s32.backward()
    clocks = Clocks(local)
    ms_grad = timed(lambda: (s32.forward(p0), s32.backward()), a.steps)
    clk = clocks.stop()
    ms_fwd = timed(lambda: s32.forward(p0), a.steps)
    mem, cg = s32.stats()
    loss32 = s32.forward(p0)
    g32 = s32.backward()
    s32.destroy()
    s64 = d.make(fp64=True, device=local)
    loss64 = s64.forward(p0)
    g64 = s64.backward()
    idx = [6, 7, 8, 15, 24, 25]
    fd = []
    for i in idx:
        e = np.zeros(27)
        e[i] = 1e-3
        fd.append((s64.forward(p0 + e, record=False) - s64.forward(p0 - e, record=False)) / 2e-3)
    fd = np.array(fd)
    s64.destroy()
    # the collider as the box's distance grid (sdfEval's trilinear sampling, its gradient and Hessian in the adjoint):
    # the FP32 gradient against the FP64 one, and its time
    g32g = g64g = None
    sg = d.make(collider="grid", device=local)
    ms_grid = timed(lambda: (sg.forward(p0), sg.backward()), 1)
    sg.forward(p0)
    g32g = sg.backward()
    sg.destroy()
    sg64 = d.make(fp64=True, collider="grid", device=local)
    sg64.forward(p0)
    g64g = sg64.backward()
    sg64.destroy()
    # the rollout against the FLIP step on the same scene (the particles' displacements and the final density splat)
    from splashtank_b200.diff import flip_rollout
    sv = d.make(collider="grid", margin=0.15 / n, cg_tol=1e-6, device=local)
    sv.forward(p0)
    xd, _ = sv.state()
    sv.destroy()
    xf = flip_rollout(d, p0, device=local)
    disp_d, disp_f = xd - d.pos, xf - d.pos
    rho_d, rho_f = scenes.splat_density(xd, n), scenes.splat_density(np.clip(xf, 0.0, 1.0), n)
    vs_flip = {"displacement_rel_l2": float(np.linalg.norm(disp_d - disp_f) / np.linalg.norm(disp_f)),
               "density_rel_l2": float(np.linalg.norm(rho_d - rho_f) / np.linalg.norm(rho_f)),
               "displacement_rms": float(np.sqrt((disp_f ** 2).sum(1).mean())),
               "flip_step": "st_flip_step on the same particles, the box's distance grid on the same keyframe path, SOR 400 "
                            "iterations, no density correction"}
    ps = d.pos.shape[0] * d.steps
    if rank == 0:
        line = {"metric": "gradient particle-steps/s (forward + adjoint)", "value": ps / (ms_grad * 1e-3), "unit": "particle-steps/s",
                "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_grad, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (f64 reference)", "data": "synthetic (seeded)",
                "config": {"workload": a.workload, "grid": [n] * 3, "particles": int(d.pos.shape[0]), "rollout_steps": d.steps,
                           "checkpoint_every": d.ckpt, "params": "8 collider keyframes (xyz) + initial velocity",
                           "collider": "analytic box, half extents 0.06 x 0.12 x 0.25", "note": "ms_per_step: one whole gradient (rollout)"},
                "forward_ms": ms_fwd, "gradient_ms": ms_grad, "device_bytes": int(mem), "cg_iterations_last": int(cg),
                "loss_f32": loss32, "loss_f64": loss64,
                "grad_check": {"f32_vs_f64_adjoint_rel_l2": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
                               "f64_adjoint_vs_fd_max_rel": float(np.max(np.abs(g64[idx] - fd)) / max(np.max(np.abs(fd)), 1e-300)),
                               "params_checked": idx, "fd_eps": 1e-3},
                "grid_collider": {"gradient_ms": ms_grid,
                                  "f32_vs_f64_adjoint_rel_l2": float(np.linalg.norm(g32g - g64g) / np.linalg.norm(g64g))},
                "vs_flip_step": vs_flip,
                "clocks": clk, "roofline": None, "gpu_launches": None,
                "e2e": {"value": ps / (ms_grad * 1e-3), "unit": "particle-steps/s", "h2d_bytes_per_step": 27 * 8, "d2h_bytes_per_step": 27 * 8,
                        "note": "parameters up and gradient back through the C ABI are inside the timed calls"},
                "cpu_baseline": None, "cpu_baseline_note": "the reference has no gradient; no CPU adjoint exists to time"}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def main():
    a = parse()
    if a.workload.startswith("pressure_"):
        return run_pressure_reference(a) if a.impl == "reference" else run_pressure(a)
    if a.workload.startswith("batch_"):
        return run_batch_reference(a) if a.impl == "reference" else run_batch(a)
    if a.workload.startswith("pbf_"):
        return run_pbf_reference(a) if a.impl == "reference" else run_pbf(a)
    if a.workload.startswith("diff_"):
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no differentiable rollout"}), flush=True)
            return None
        return run_diff(a)
    if a.impl == "reference":
        return run_reference(a)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    w = workload(a.workload)
    sim = w.make(FlipSim, device=local)
    run = SceneRunner(sim)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    t = 0.0

    def step():
        nonlocal t
        t += w.dt
        run.step(w.dt, w.states(t), w.opts)

    # the stage timer is on from the first warm-up step, so the timed steps' graph (with its event nodes) is captured
    # and instantiated before the timed region; the warm-up's stage times are read and discarded
    sim.set_timing(True)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    sim.read_timing()
    st0 = sim.readStats()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed region
    clocks = Clocks(local)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    stages, nrec = sim.read_timing()
    sim.set_timing(False)
    st1 = sim.readStats()
    live = st1["live"]
    launches = st1["launches"] - st0["launches"]
    ms_max, live_sum = ms, live
    if dist:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
        tl = torch.tensor([float(live)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tl)
        live_sum = int(tl.item())
    value = live_sum * a.steps / (ms_max * 1e-3)

    # ---- end to end through the C ABI with host buffers: every step the options and collider records go up from pinned
    # host memory and the step's counters come back (readStats as the reference issues it: queued behind the step,
    # waited for once the next step is queued, so the device never idles while the host reads them); every 4th step (a
    # 60 Hz frame at dt 1/240) the particles come back as a cache frame (6 + 1 + 1 bytes per point, packed on the device)
    # into pinned host memory, as a bake stores them: st_flip_read_frame_async, so the copy runs while the next steps
    # compute, and st_flip_frame_wait before the next frame and at the end (inside the timed region)
    n_all = st1["n"]
    cap = max(sim.MAXN, 1)
    pin = torch.empty(cap * 8, dtype=torch.uint8, pin_memory=True).numpy()
    fbuf = (pin[:cap * 6].view(np.uint16).reshape(cap, 3), pin[cap * 6:cap * 7], pin[cap * 7:cap * 8])
    nc = len(w.states(0.0))
    h2d = 496 + nc * 128   # the 496-byte parameter block and 128 bytes per collider record, per step
    d2h = 64 + (8 * n_all) / 4.0
    if a.no_e2e:
        a.e2e_steps = 0

    def e2e_run(steps):
        prev = None
        for k in range(steps):
            step()
            tk = sim.readStatsAsync()
            if prev is not None:
                sim.statsWait(prev)
            prev = tk
            if k % 4 == 3:
                sim.frame_wait()
                sim.read_frame_async(1.0, out=fbuf)
        if prev is not None:
            sim.statsWait(prev)
        sim.frame_wait()

    if a.e2e_steps:
        e2e_run(8)   # untimed: the copy stream, the pinned frame buffer and the counter ring get their first use
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    e2e_run(a.e2e_steps)
    f1.record(stream)
    f1.synchronize()
    barrier()
    ems = f0.elapsed_time(f1)
    if dist:
        tt = torch.tensor([ems], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ems = float(tt.item())
    e2e_value = live_sum * a.e2e_steps / (ems * 1e-3) if a.e2e_steps else None

    if rank == 0:
        peak, src = measured_peak()
        cells = st1["sc"] * 512
        iters = w.opts.get("iters", 30)
        rl = roofline(stages, nrec, live, cells, st1["fluid"], iters, peak, src)
        nb_on = bool(w.opts.get("nb", {}).get("on"))
        ww = min(st1["spray_used"], w.spray_cap) if w.spray_cap else None
        srl = step_roofline(ms / a.steps, live, cells, st1["fluid"], iters, nb_on, ww, stages, nrec, peak, src)
        if rl is not None:
            rl.update(srl)
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded jitter, 8 particles per cell)",
                "config": config_of(a.workload, w, live), "gpu_launches": int(launches),
                "stage_ms_per_step": {k: round(v / max(nrec, 1), 4) for k, v in stages.items()},
                "clocks": clk, "roofline": rl,
                "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                        "steps": a.e2e_steps, "readback": "counters every step (read once the next step is queued), a packed cache frame of all particles every 4th step, copied while the next steps run"}}
        if world == 1:
            sim.destroy()
            del sim
            if not a.no_extras and a.workload.startswith("wave_tank"):
                # the metric's pressure half, the reference's narrow band of 3 cells, config 2 with its PBF stage, and the
                # batching and differentiation configurations, after the timed regions
                line["pressure"] = pressure_summary(local)
                line["band3"] = band_summary(local, a.workload + "_band3")
                line["pbf4"] = pbf4_summary(local, a.workload)
                # config 2 with everything it names at once: the 3-cell narrow band and the 4-iteration PBF stage
                line["band3_pbf4"] = pbf4_summary(local, a.workload + "_band3", warm=8, steps=20)
                line["batch64"] = batch_summary(local)
                line["diff128"] = diff_summary(local)
            if not a.no_cpu_baseline:
                cb, _ = cpu_sample(a.workload, w)
                line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
