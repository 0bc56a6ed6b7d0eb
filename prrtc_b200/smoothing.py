"""Post-plan path smoothing with the hand-written adjoint kernel.

``SmoothCost`` is a ``torch.autograd.Function`` whose forward and backward both
come from ``prrtc_b200_smooth_cost_grad`` (one launch computes the cost and the
gradient through FK, recomputing link transforms instead of storing them) -- the
torch counterpart of a ``jax.custom_vjp`` (jax is not installed here).

Cost of a path with W waypoints q_w:
    sum_w sum_pairs softplus_beta(margin - d_pair(q_w)) + w_len * sum_w |q_{w+1} - q_w|^2
over every robot-sphere / world-primitive pair and every self pair.

``smooth_paths`` runs projected gradient steps (endpoints fixed, joint limits
enforced), then re-validates every smoothed path with the exact collision
checker at a fixed joint-space resolution; a path that fails reverts to the
input path (prrtc_plan's RRT-Connect result).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .collision import CollisionChecker
from .device import DeviceContext, as_tensor, cuda_device, ptr, stream_handle, workspace


class SmoothContext:
    """Robot + world tables resident on the device for the smoothing kernel."""

    def __init__(self, collision_context: dict, dim: int, margin: float = 0.02, beta: float = 50.0,
                 w_len: float = 1.0, device=None):
        self.lib = _lib.load()
        self.device = cuda_device(device)
        self.ctx = DeviceContext(collision_context, self.device)
        self.dim = int(dim)
        self.margin, self.beta, self.w_len = float(margin), float(beta), float(w_len)
        self.robot, self.world = self.ctx.robot(), self.ctx.world()
        self.ws = workspace(self.lib.prrtc_b200_smooth_workspace_size(C.byref(self.robot), C.byref(self.world)),
                            self.device)

    def cost_grad(self, waypoints: torch.Tensor, need_grad: bool = True):
        wp = waypoints.detach().to(self.device, torch.float32).contiguous()
        P, W, dim = wp.shape
        cost = torch.empty((P,), dtype=torch.float32, device=self.device)
        grad = torch.empty_like(wp) if need_grad else None
        _lib.check(self.lib.prrtc_b200_smooth_cost_grad(C.byref(self.robot), C.byref(self.world), dim, ptr(wp), P, W,
                                                        self.margin, self.beta, self.w_len, ptr(cost), ptr(grad),
                                                        self.ws.data_ptr(), self.ws.numel(), stream_handle()),
                   "prrtc_b200_smooth_cost_grad")
        return cost, grad


class SmoothCost(torch.autograd.Function):
    """cost[P] = smooth collision + length cost of waypoints [P, W, dim]."""

    @staticmethod
    def forward(ctx, waypoints, sctx: SmoothContext):
        cost, grad = sctx.cost_grad(waypoints, need_grad=waypoints.requires_grad)
        ctx.save_for_backward(grad if grad is not None else torch.empty(0))
        return cost

    @staticmethod
    def backward(ctx, gcost):
        (grad,) = ctx.saved_tensors
        return grad * gcost[:, None, None], None


def smooth_cost(waypoints: torch.Tensor, sctx: SmoothContext) -> torch.Tensor:
    return SmoothCost.apply(waypoints, sctx)


def resample_path(path: np.ndarray, W: int) -> np.ndarray:
    """W waypoints evenly spaced in arc length along a piecewise-linear path."""
    path = np.asarray(path, dtype=np.float64)
    if path.shape[0] == 1:
        return np.repeat(path, W, 0).astype(np.float32)
    seg = np.linalg.norm(np.diff(path, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    if s[-1] <= 0:
        return np.repeat(path[:1], W, 0).astype(np.float32)
    t = np.linspace(0.0, s[-1], W)
    idx = np.clip(np.searchsorted(s, t, side="right") - 1, 0, path.shape[0] - 2)
    u = ((t - s[idx]) / np.maximum(seg[idx], 1e-12))[:, None]
    out = path[idx] * (1 - u) + path[idx + 1] * u
    out[0], out[-1] = path[0], path[-1]
    return out.astype(np.float32)


def densify(paths: torch.Tensor, resolution: float) -> tuple[torch.Tensor, torch.Tensor]:
    """Points every <= `resolution` (joint-space L2) along each polyline [P, W, dim];
    returns configs [M, dim] and the path index of each point."""
    P, W, dim = paths.shape
    d = torch.linalg.norm(paths[:, 1:] - paths[:, :-1], dim=-1)           # [P, W-1]
    n = torch.clamp(torch.ceil(d / resolution), min=1).to(torch.int64)    # [P, W-1]
    n_cpu = n.cpu().numpy()
    pts, owner = [], []
    for p in range(P):
        for w in range(W - 1):
            k = int(n_cpu[p, w])
            t = torch.arange(0, k + 1 if w == W - 2 else k, device=paths.device, dtype=paths.dtype) / k
            pts.append(paths[p, w][None] + t[:, None] * (paths[p, w + 1] - paths[p, w])[None])
            owner.append(torch.full((t.shape[0],), p, device=paths.device, dtype=torch.int64))
    return torch.cat(pts, 0), torch.cat(owner, 0)


def smooth_paths(paths: list, collision_context: dict, lower, upper, *, waypoints: int = 64, steps: int = 50,
                 lr: float = 0.05, margin: float = 0.02, beta: float = 50.0, w_len: float = 1.0,
                 resolution: float = 0.01, device=None):
    """Smooth each path (list of [L_i, dim] arrays) with projected gradient steps
    on the adjoint cost; re-validate at `resolution`; revert paths that fail.

    Returns (smoothed [P, waypoints, dim] tensor, accepted [P] bool tensor,
    cost before [P], cost after [P])."""
    dev = cuda_device(device)
    dim = int(np.asarray(paths[0]).shape[1])
    init = torch.from_numpy(np.stack([resample_path(p, waypoints) for p in paths])).to(dev)
    lo = as_tensor(lower, torch.float32, dev).reshape(1, 1, dim)
    hi = as_tensor(upper, torch.float32, dev).reshape(1, 1, dim)
    sctx = SmoothContext(collision_context, dim, margin, beta, w_len, dev)
    x = init.clone()
    mask = torch.ones_like(x)
    mask[:, 0] = 0.0
    mask[:, -1] = 0.0
    c0, _ = sctx.cost_grad(init, need_grad=False)
    for _ in range(steps):
        _, g = sctx.cost_grad(x)
        # normalised step per path keeps the update scale independent of the cost scale
        gn = torch.linalg.norm((g * mask).reshape(g.shape[0], -1), dim=1).clamp_min(1e-12)
        x = torch.minimum(torch.maximum(x - lr * (g * mask) / gn[:, None, None], lo), hi)
    c1, _ = sctx.cost_grad(x, need_grad=False)
    checker = CollisionChecker(collision_context, dim, "binary", 0.0, dev)
    pts, owner = densify(x, resolution)
    v = checker.check(pts).to(torch.int64)
    bad = torch.zeros((x.shape[0],), dtype=torch.int64, device=dev).index_add_(0, owner, v)
    accepted = bad == 0
    out = torch.where(accepted[:, None, None], x, init)
    return out, accepted, c0, c1
