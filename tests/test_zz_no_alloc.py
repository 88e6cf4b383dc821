"""st_poisson_residual_noalloc: the pressure residual on caller-owned device arrays with a fixed device scratch array,
against the residual st_poisson_solve reports for the same solution. Named to be collected last."""
import numpy as np
import pytest

from splashtank_b200 import scenes


@pytest.mark.gpu
def test_residual_noalloc_matches_solve_on_consecutive_calls():
    import torch
    from splashtank_b200 import abi, poisson
    from splashtank_b200.flip import StError
    n = 48
    ty, b = scenes.splash_blobs(n, seed=7)
    g = poisson.PoissonSolver((n, n, n))
    g.set(ty, b)
    r = g.solve(poisson.REFINE, tol=1e-6, omega=1.9, inner_sweeps=40, max_sweeps=20000)
    x = g.read()
    g.destroy()
    tiles, info, bt = poisson.tile_system(ty, b)
    dev = torch.device("cuda", 0)
    T = torch.from_numpy(tiles.view(np.int32)).to(dev)
    I = torch.from_numpy(info.view(np.int16)).to(dev)
    B = torch.from_numpy(bt).to(dev)
    X = torch.from_numpy(poisson.to_tile_major(x)).to(dev)
    Z = torch.zeros_like(X)
    torch.cuda.synchronize()
    tol = 1e-12   # same per-tile tree and tile-order sum as the solve's own norm: equal up to rounding
    for _ in range(2):
        rel, r2, b2 = poisson.residual_noalloc((n, n, n), T, I, B, X)
        assert abs(rel - r["rel_residual"]) <= tol * r["rel_residual"], (rel, r["rel_residual"])
        rel0, r20, b20 = poisson.residual_noalloc((n, n, n), T, I, B, Z)
        assert abs(rel0 - 1.0) <= tol and b20 == b2 and r20 == b20
    # more tiles than the fixed scratch holds: rejected before any launch
    big = abi.NOALLOC_MAX_TILES + 1

    class Fake:
        def __init__(self, t, k):
            self.t, self.k = t, k

        def numel(self):
            return self.k

        def data_ptr(self):
            return self.t.data_ptr()
    with pytest.raises(StError, match="exceeds the fixed scratch of 65536 tiles"):
        poisson.residual_noalloc((1024, 1024, 1024), Fake(T, big), I, B, X)
    rel, _, _ = poisson.residual_noalloc((n, n, n), T, I, B, X)
    assert abs(rel - r["rel_residual"]) <= tol * r["rel_residual"]
