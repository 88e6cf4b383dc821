"""Many tanks per step (st_batch_*): the tank set, the split over GPUs, and on the GPU the same result as stepping
each tank alone, in one graph launch and sequentially."""
import os

import numpy as np
import pytest

from splashtank_b200 import scenes
from splashtank_b200.batch import lpt_partition


def test_batch_tanks_follow_the_spec():
    b = scenes.BatchTanks()
    assert len(b.tanks) == 64
    for t in b.tanks:
        assert all(e in scenes.TANK_EDGES for e in t["edges"])
        f = t["fill"][0] * t["fill"][1] * t["fill"][2]
        assert 0.2 <= f <= 0.6 + 1e-12 and all(0 < a <= 1 for a in t["fill"])
        assert all(0 <= lo <= 1 - a + 1e-12 for lo, a in zip(t["lo"], t["fill"]))
    again = scenes.BatchTanks()
    assert [t["edges"] for t in again.tanks] == [t["edges"] for t in b.tanks]
    p = b.particles(3)
    assert np.array_equal(p, again.particles(3))
    t = b.tanks[3]
    lo = np.array([-t["size"][0] / 2, 0.0, -t["size"][2] / 2])
    assert np.all(p >= lo) and np.all(p <= lo + np.array(t["size"]))


def test_lpt_partition_covers_every_tank_once_and_balances():
    b = scenes.BatchTanks()
    costs = [b.cost(k) for k in range(64)]
    for parts in (1, 2, 3, 8):
        split = lpt_partition(costs, parts)
        flat = sorted(i for s in split for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in split]
        # LPT: no part exceeds the mean by more than the largest task
        assert max(loads) <= sum(costs) / parts + max(costs) + 1e-9
        assert split == lpt_partition(costs, parts)


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = scenes.BatchTanks()
    mine = lpt_partition([b.cost(k) for k in range(64)], world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    # the bench's reduction: slowest rank's time, total particles
    t = torch.tensor([10.0 + rank])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(len(mine))])
    dist.all_reduce(n)
    if rank == 0:
        out.put((got, float(t.item()), float(n.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_tanks_split_over_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got, tmax, n = q.get(timeout=120)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    assert sorted(got[0] + got[1]) == list(range(64)) and not set(got[0]) & set(got[1])
    assert tmax == 11.0 and n == 64.0


@pytest.mark.gpu
def test_batch_step_matches_single_tank_steps():
    from splashtank_b200.batch import TankBatch
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    spec = scenes.BatchTanks(count=4, seed=9, edges=(32, 48))
    runs = {}
    for mode in ("graph", "sequential", "pooled", "persistent", "single"):
        made = [spec.make(k, FlipSim) for k in range(4)]
        sims = [m[0] for m in made]
        runners = [SceneRunner(s) for s in sims]
        if mode in ("graph", "pooled"):
            sims[1].set_launch(2, 1, 2)   # launch shapes differ per tank; results must not
        batch = TankBatch(sims, mode) if mode != "single" else None
        if mode == "persistent":
            batch.set_sweeps(2)
        for _ in range(6):
            opts = [spec.step_opts(k, sims[k], runners[k]) for k in range(4)]
            if batch:
                batch.step(spec.dt, opts)
            else:
                for k in range(4):
                    sims[k].step(spec.dt, opts[k])
        out = []
        for s in sims:
            dst = np.zeros((s.MAXN, 4), np.float32)
            n = s.readbackInto(dst)
            out.append(dst[:n].copy())
        runs[mode] = out
        if batch:
            assert batch.launches() > 0
            batch.destroy()
        for s in sims:
            s.destroy()
    for k in range(4):
        for mode in ("graph", "sequential", "pooled", "persistent"):
            assert np.array_equal(runs[mode][k].view(np.uint32), runs["single"][k].view(np.uint32)), (mode, k)


@pytest.mark.gpu
def test_persistent_sweep_barrier_wait_is_bounded():
    """The persistent sweep's grid barrier with one CTA that never arrives: every wait runs out after its limit, the
    kernel sets its error flag and returns, and the device stays usable (a batch step runs right after)."""
    import time
    from splashtank_b200.batch import TankBatch, barrier_test
    from splashtank_b200.flip import FlipSim
    from splashtank_b200.scene import SceneRunner
    t0 = time.perf_counter()
    assert barrier_test(missing=1, limit_us=200_000)
    assert time.perf_counter() - t0 < 20.0
    spec = scenes.BatchTanks(count=2, seed=3, edges=(32,))
    sims = [spec.make(k, FlipSim)[0] for k in range(2)]
    runners = [SceneRunner(s) for s in sims]
    b = TankBatch(sims, "persistent")
    for _ in range(3):
        b.step(spec.dt, [spec.step_opts(k, sims[k], runners[k]) for k in range(2)])
    assert all(s.readStats()["steps"] == 3 for s in sims)
    b.destroy()
    for s in sims:
        s.destroy()
