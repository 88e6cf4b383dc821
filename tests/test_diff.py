"""Differentiable rollout (st_diff_*): the hand-written adjoint against central finite differences of the frozen FP64
forward pass (eps 1e-3), the FP32 adjoint against the FP64 one, and the torch.autograd.Function wrapper."""
import numpy as np
import pytest

from splashtank_b200 import scenes


def test_target_splat_conserves_particles():
    d = scenes.DiffDam(n=16, steps=4, ckpt=2)
    assert abs(d.target.sum() - len(d.pos)) < 1e-3 * len(d.pos)
    assert d.params.shape == (27,) and np.all(d.pos >= 0) and np.all(d.pos <= 1)


def small(fp64):
    d = scenes.DiffDam(n=24, steps=6, ckpt=3, seed=5)
    return d, d.make(fp64=fp64, box_half=(0.1, 0.15, 0.3))


@pytest.mark.gpu
def test_adjoint_matches_fp64_central_differences():
    d, s = small(True)
    p0 = d.params.copy()
    # move the collider into the water so its keyframes matter
    p0[:24] = np.array([[0.55 - 0.02 * k, 0.25, 0.5] for k in range(8)]).ravel()
    p0[24:] = [0.5, 0.1, 0.0]
    s.forward(p0, record=True)
    g = s.backward()

    def fd(eps):
        out = np.zeros(27)
        for i in range(27):
            e = np.zeros(27)
            e[i] = eps
            out[i] = (s.forward(p0 + e, record=False) - s.forward(p0 - e, record=False)) / (2 * eps)
        return out
    # eps 1e-3 (2.4% of a cell here): the trilinear weights are piecewise linear in the positions, so particles that
    # cross a cell face within the difference bend the secant; the error shrinks with eps while the adjoint stays put
    f3 = fd(1e-3)
    assert np.linalg.norm(g - f3) <= 3e-2 * np.linalg.norm(f3), (g, f3)
    f6 = fd(1e-6)
    # at eps 1e-6 a rare crossing can still bend one component; the rest agree to about 1e-5
    assert np.linalg.norm(g - f6) <= 1e-3 * np.linalg.norm(f6), (g, f6)
    assert np.median(np.abs(g - f6) / np.maximum(np.abs(f6), 1e-9 * np.abs(f6).max())) <= 1e-4, (g, f6)
    assert np.linalg.norm(g - f6) < np.linalg.norm(g - f3)
    assert np.any(np.abs(g[:24]) > 1e-3 * np.abs(f6).max())   # the collider keyframes do get a gradient
    s.destroy()


@pytest.mark.gpu
def test_fp32_adjoint_close_to_fp64():
    d, s64 = small(True)
    _, s32 = small(False)
    p0 = d.params.copy()
    p0[:24] = np.array([[0.55 - 0.02 * k, 0.25, 0.5] for k in range(8)]).ravel()
    l64 = s64.forward(p0)
    l32 = s32.forward(p0)
    assert abs(l32 - l64) <= 1e-3 * l64
    g64, g32 = s64.backward(), s32.backward()
    assert np.linalg.norm(g32 - g64) <= 2e-2 * np.linalg.norm(g64), (g32, g64)


@pytest.mark.gpu
def test_torch_autograd_function_wraps_the_adjoint():
    import torch

    d, s = small(True)

    class Rollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params):
            return torch.tensor(s.forward(params.detach().cpu().numpy(), record=True), dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            return torch.from_numpy(s.backward()) * gout

    prm = torch.tensor(d.params, dtype=torch.float64, requires_grad=True)
    loss = Rollout.apply(prm)
    loss.backward()
    s.forward(d.params, record=True)
    assert torch.allclose(prm.grad, torch.from_numpy(s.backward()), rtol=1e-12, atol=0)
    # a small step against the gradient lowers the loss (the same discrete decisions held)
    gr = prm.grad.numpy()
    step = 1e-4 / np.abs(gr).max()
    assert s.forward(d.params - step * gr, record=False) < float(loss.detach())
