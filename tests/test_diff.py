"""Differentiable rollout (st_diff_*): the hand-written adjoint against central finite differences of the frozen FP64
forward pass (eps 1e-3), the FP32 adjoint against the FP64 one, and the torch.autograd.Function wrapper."""
import numpy as np
import pytest

from splashtank_b200 import scenes


def test_target_splat_conserves_particles():
    d = scenes.DiffDam(n=16, steps=4, ckpt=2)
    assert abs(d.target.sum() - len(d.pos)) < 1e-3 * len(d.pos)
    assert d.params.shape == (27,) and np.all(d.pos >= 0) and np.all(d.pos <= 1)


def small(fp64, collider="box"):
    d = scenes.DiffDam(n=24, steps=6, ckpt=3, seed=5)
    return d, d.make(fp64=fp64, box_half=(0.1, 0.15, 0.3), collider=collider)


def _fd(s, p0, eps):
    out = np.zeros(27)
    for i in range(27):
        e = np.zeros(27)
        e[i] = eps
        out[i] = (s.forward(p0 + e, record=False) - s.forward(p0 - e, record=False)) / (2 * eps)
    return out


def _contact_params(d):
    p0 = d.params.copy()
    # move the collider into the water so its keyframes matter
    p0[:24] = np.array([[0.55 - 0.02 * k, 0.25, 0.5] for k in range(8)]).ravel()
    p0[24:] = [0.5, 0.1, 0.0]
    return p0


@pytest.mark.gpu
def test_adjoint_matches_fp64_central_differences():
    """The collider as the box's distance grid, sampled as the step samples a collider grid (sdfEval: trilinear distance,
    normalised trilinear gradient) and differentiated through that gradient and its Hessian, with the step's velocity
    response to the push-out and the wall clamp: the FP64 adjoint against FP64 central differences of the frozen
    forward pass. At the requested eps 1e-3 (2.4% of a cell here) particles that cross a face where the trilinear
    weights bend, or pass the collider's surface, bend the secant: within 1%; at eps 1e-7 within 1e-3, with the median
    component to 1e-4."""
    d, s = small(True, "grid")
    p0 = _contact_params(d)
    s.forward(p0, record=True)
    g = s.backward()
    f3 = _fd(s, p0, 1e-3)
    assert np.linalg.norm(g - f3) <= 1e-2 * np.linalg.norm(f3), (np.linalg.norm(g - f3) / np.linalg.norm(f3), g, f3)
    f7 = _fd(s, p0, 1e-7)
    assert np.linalg.norm(g - f7) <= 1e-3 * np.linalg.norm(f7), (g, f7)
    assert np.median(np.abs(g - f7) / np.maximum(np.abs(f7), 1e-9 * np.abs(f7).max())) <= 1e-4, (g, f7)
    assert np.any(np.abs(g[:24]) > 1e-3 * np.abs(f7).max())   # the collider keyframes do get a gradient
    s.destroy()


@pytest.mark.gpu
def test_adjoint_with_the_analytic_box_at_small_eps():
    """The analytic box collider (exact distance, its gradient and Hessian): against FP64 central differences at eps
    1e-6, where few particles cross a kink of the frozen function (at 1e-3 the box's surface, which the collider's
    keyframes move through the water, bends the secant by tens of percent)."""
    d, s = small(True, "box")
    p0 = _contact_params(d)
    s.forward(p0, record=True)
    g = s.backward()
    f6 = _fd(s, p0, 1e-6)
    assert np.linalg.norm(g - f6) <= 2e-3 * np.linalg.norm(f6), (g, f6)
    assert np.median(np.abs(g - f6) / np.maximum(np.abs(f6), 1e-9 * np.abs(f6).max())) <= 1e-4, (g, f6)
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
    # the same recording differentiated again outside autograd: the adjoint's sums are FP64 atomics (order-dependent in
    # the last bits), so the two agree to rounding, not bits. A second recording is not compared: a particle that slides
    # along the collider has v.n at rounding level after the push-out, so the atomic order can flip its recorded contact
    # decision and with it a small gradient component.
    assert torch.allclose(prm.grad, torch.from_numpy(s.backward()), rtol=1e-6, atol=1e-9 * float(prm.grad.abs().max()))
    # a small step against the gradient lowers the loss (the same discrete decisions held)
    gr = prm.grad.numpy()
    step = 1e-4 / np.abs(gr).max()
    assert s.forward(d.params - step * gr, record=False) < float(loss.detach())


@pytest.mark.gpu
@pytest.mark.parametrize("contact", [False, True])
def test_rollout_tracks_the_flip_step(contact):
    """The differentiable rollout against st_flip_step on the differentiation workload's scene (the dam break with the
    moving box collider, at 32^3 for 16 steps): the same particles and keyframed collider path through the FLIP step,
    whose collider is the same distance grid (its SOR run for 400 iterations, no density correction). Without contact
    they differ only by the fixed-point P2G and the unconverged SOR against conjugate gradients; with the collider
    driven into the water, also by the frozen collider cells and the float sums: the particles' displacements and the
    final density splat stay within 1e-3 and 3e-2 of the step's."""
    from splashtank_b200.diff import flip_rollout
    n, steps = 32, 16
    d = scenes.DiffDam(n=n, steps=steps, ckpt=8)
    p0 = d.params.copy()
    if contact:
        p0[:24] = np.array([[0.5 - 0.02 * k, 0.25, 0.5] for k in range(8)]).ravel()
    s = d.make(fp64=False, collider="grid", margin=0.15 / n, cg_tol=1e-6)
    s.forward(p0, record=True)
    xd, _ = s.state()
    s.destroy()
    xf = flip_rollout(d, p0)
    disp_d, disp_f = xd - d.pos, xf - d.pos
    rel = np.linalg.norm(disp_d - disp_f) / np.linalg.norm(disp_f)
    rd, rf = scenes.splat_density(xd, n), scenes.splat_density(np.clip(xf, 0.0, 1.0), n)
    rho_rel = np.linalg.norm(rd - rf) / np.linalg.norm(rf)
    assert np.sqrt((disp_f ** 2).sum(1).mean()) > 0.5 / n       # the water moved by more than half a cell
    bound = 3e-2 if contact else 1e-3
    assert rel < bound and rho_rel < bound, (rel, rho_rel)
