"""Adjoint smoothing kernel: cost against the float64 oracle, gradient against
central finite differences (h = 1e-3) of the oracle cost and against
torch.autograd of a float64 restatement of the cost, the autograd wrapper,
and the smoothing pass (accepted paths re-validate, rejected ones revert)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import make_problem

pytestmark = pytest.mark.gpu

MARGIN, BETA, WLEN = 0.02, 50.0, 1.0


def _solved_path(orc, kind, seed):
    pr = make_problem(kind, seed)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=3000, num_new_samples=32,
                 max_nodes=16384, collision_mode=3, edge_resolution=0.01)
    assert r.solved == 1
    return pr, sc, r.path


def _fd_grad(sc, w, h=1e-3):
    g = np.zeros_like(w)
    for i in range(w.shape[0]):
        for d in range(w.shape[1]):
            wp, wm = w.copy(), w.copy()
            wp[i, d] += h
            wm[i, d] -= h
            g[i, d] = (sc.smooth_cost(wp, MARGIN, BETA, WLEN) - sc.smooth_cost(wm, MARGIN, BETA, WLEN)) / (2 * h)
    return g


@pytest.mark.parametrize("kind,seed", [("tabletop", 3), ("spheres16", 1), ("uneven", 7)])
def test_adjoint_matches_finite_differences(cuda, orc, kind, seed):
    from prrtc_b200.smoothing import SmoothContext, resample_path

    pr, sc, path = _solved_path(orc, kind, seed)
    w = resample_path(path, 16)
    sctx = SmoothContext(pr.context, pr.dim, MARGIN, BETA, WLEN, cuda)
    cost, grad = sctx.cost_grad(torch.from_numpy(w)[None].to(cuda))
    c64 = sc.smooth_cost(w.astype(np.float64), MARGIN, BETA, WLEN)
    assert abs(cost.item() - c64) <= 1e-4 * max(1.0, abs(c64))
    g_fd = _fd_grad(sc, w.astype(np.float64))
    g = grad[0].cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(g - g_fd) / np.linalg.norm(g_fd)
    assert rel < 1e-3, rel


@pytest.mark.parametrize("kind,seed", [("tabletop", 3), ("spheres16", 1), ("uneven", 7)])
def test_adjoint_matches_autodiff_reference(cuda, orc, kind, seed):
    """The adjoint kernel against torch.autograd of a float64 restatement of
    the same cost (oracle/smooth_autodiff.py), the stand-in for jax.grad of a
    pure-JAX FK + SDF reference (jax is not installed: the jax check is not
    run).  Tolerance as for the central differences: 1e-3 relative."""
    from oracle.smooth_autodiff import smooth_grad
    from prrtc_b200.smoothing import SmoothContext, resample_path

    pr, sc, path = _solved_path(orc, kind, seed)
    w = resample_path(path, 16)
    sctx = SmoothContext(pr.context, pr.dim, MARGIN, BETA, WLEN, cuda)
    cost, grad = sctx.cost_grad(torch.from_numpy(w)[None].to(cuda))
    c_ad, g_ad = smooth_grad(pr.context, w.astype(np.float64), MARGIN, BETA, WLEN)
    assert abs(cost.item() - c_ad) <= 1e-4 * max(1.0, abs(c_ad))
    g = grad[0].cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(g - g_ad) / np.linalg.norm(g_ad)
    assert rel < 1e-3, rel


def test_autograd_function_and_batch(cuda, orc):
    from prrtc_b200.smoothing import SmoothContext, resample_path, smooth_cost

    pr, sc, path = _solved_path(orc, "tabletop", 4)
    w = torch.from_numpy(np.stack([resample_path(path, 64)] * 3)).to(cuda)
    w[1] += 0.01
    sctx = SmoothContext(pr.context, pr.dim, MARGIN, BETA, WLEN, cuda)
    x = w.clone().requires_grad_(True)
    c = smooth_cost(x, sctx)
    (c * torch.tensor([1.0, 2.0, 0.5], device=cuda)).sum().backward()
    _, g = sctx.cost_grad(w)
    assert torch.allclose(x.grad[0], g[0], rtol=1e-5, atol=1e-6)
    assert torch.allclose(x.grad[1], 2.0 * g[1], rtol=1e-5, atol=1e-6)
    assert torch.allclose(x.grad[2], 0.5 * g[2], rtol=1e-5, atol=1e-6)
    for p in range(3):
        c64 = sc.smooth_cost(w[p].cpu().numpy().astype(np.float64), MARGIN, BETA, WLEN)
        assert abs(c[p].item() - c64) <= 1e-4 * max(1.0, abs(c64))


def test_smoothing_pass_revalidates_or_reverts(cuda, orc):
    from prrtc_b200.smoothing import smooth_paths

    probs = [_solved_path(orc, "tabletop", s) for s in (10, 11, 12, 13)]
    ctx = probs[0][0].context
    # same world for all paths: plan each problem's start/goal in problem 0's world
    paths = []
    sc0 = probs[0][1]
    for pr, _, _ in probs:
        r = orc.plan(sc0, pr.start if sc0.in_collision(pr.start) is False else probs[0][0].start,
                     probs[0][0].goals, pr.lower, pr.upper, max_iterations=3000, num_new_samples=32,
                     max_nodes=16384, collision_mode=3, edge_resolution=0.01)
        if r.solved == 1:
            paths.append(r.path)
    assert paths
    out, accepted, c0, c1 = smooth_paths(paths, ctx, probs[0][0].lower, probs[0][0].upper, waypoints=64, steps=50)
    out = out.cpu().numpy()
    for p in range(len(paths)):
        ok, md = sc0.validate_path(out[p], 0.01)
        assert ok, (p, md)                       # accepted paths re-validate; rejected ones reverted
        assert np.allclose(out[p][0], paths[p][0]) and np.allclose(out[p][-1], paths[p][-1])
    assert bool(accepted.any())
    assert bool((c1[accepted] <= c0[accepted] + 1e-3).all())


def test_adjoint_mimic_dual_arm(cuda, orc):
    """The adjoint through mimic joints (the dual arm: 14 actuated values, 18
    joints, four mimic finger joints) against torch.autograd of the float64
    restatement, on a straight-line path with small perturbations."""
    from oracle.smooth_autodiff import smooth_grad
    from prrtc_b200.smoothing import SmoothContext

    pr = make_problem("large", 5)
    rng = np.random.default_rng(5)
    w = (np.linspace(pr.start, pr.goals[0], 12) + rng.normal(0, 0.03, (12, pr.dim))).astype(np.float32)
    sctx = SmoothContext(pr.context, pr.dim, MARGIN, BETA, WLEN, cuda)
    cost, grad = sctx.cost_grad(torch.from_numpy(w)[None].to(cuda))
    c_ad, g_ad = smooth_grad(pr.context, w.astype(np.float64), MARGIN, BETA, WLEN)
    assert abs(cost.item() - c_ad) <= 1e-4 * max(1.0, abs(c_ad))
    g = grad[0].cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(g - g_ad) / np.linalg.norm(g_ad)
    assert rel < 1e-3, rel


def test_batched_adjoint_each_path_in_its_own_world(cuda, orc):
    """prrtc_b200_smooth_cost_grad_batch: path p against problem p's world (the
    worlds differ in obstacle counts, so the packed tables are padded) gives the
    cost and gradient of the single-scene entry point on that world, and the
    cost of the float64 oracle; then the batched smoothing pass keeps only
    paths that re-validate in their own world, and a reverted path is the
    planner's path itself."""
    from prrtc_b200.smoothing import BatchSmoothContext, SmoothContext, resample_path, smooth_paths_batch

    cases = [_solved_path(orc, kind, seed) for kind, seed in (("tabletop", 3), ("uneven", 7), ("spheres16", 1),
                                                            ("uneven", 11))]
    W = 24
    wps = np.stack([resample_path(path, W) for _, _, path in cases])
    bctx = BatchSmoothContext([pr.context for pr, _, _ in cases], 7, MARGIN, BETA, WLEN, cuda)
    cost_b, grad_b = bctx.cost_grad(torch.from_numpy(wps).to(cuda))
    for i, (pr, sc, _) in enumerate(cases):
        one = SmoothContext(pr.context, pr.dim, MARGIN, BETA, WLEN, cuda)
        c1, g1 = one.cost_grad(torch.from_numpy(wps[i:i + 1]).to(cuda))
        assert abs(cost_b[i].item() - c1.item()) <= 1e-5 * max(1.0, abs(c1.item())), i
        assert torch.allclose(grad_b[i], g1[0], rtol=1e-5, atol=1e-6), i
        c64 = sc.smooth_cost(wps[i].astype(np.float64), MARGIN, BETA, WLEN)
        assert abs(cost_b[i].item() - c64) <= 1e-4 * max(1.0, abs(c64)), i
    pr0 = cases[0][0]
    out, acc, c0, c1 = smooth_paths_batch([path for _, _, path in cases], [pr.context for pr, _, _ in cases],
                                          pr0.lower, pr0.upper, waypoints=32, steps=20, device=cuda)
    for i, (pr, sc, path) in enumerate(cases):
        ok, _ = sc.validate_path(out[i].cpu().numpy(), 0.01)
        assert ok, i
        if not bool(acc[i]):
            assert np.array_equal(out[i].cpu().numpy(), resample_path(path, 32))
