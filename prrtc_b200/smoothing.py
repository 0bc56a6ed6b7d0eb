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
    """W waypoints along a piecewise-linear path of L vertices.  With L <= W every
    vertex is kept and the W - L extra points are spread over the segments in
    proportion to their lengths (largest remainders first), so the resampled
    polyline is the input path itself -- a smoothing pass that reverts returns
    exactly the planner's path.  With L > W: W points evenly spaced in arc
    length."""
    path = np.asarray(path, dtype=np.float64)
    if path.shape[0] == 1:
        return np.repeat(path, W, 0).astype(np.float32)
    L = path.shape[0]
    if L <= W:
        seg = np.linalg.norm(np.diff(path, axis=0), axis=1)
        extra = W - L
        share = seg / seg.sum() * extra if seg.sum() > 0 else np.full(L - 1, extra / (L - 1))
        n = np.floor(share).astype(np.int64)
        rest = extra - int(n.sum())
        if rest > 0:
            n[np.argsort(-(share - n), kind="stable")[:rest]] += 1
        out = [path[i] + (np.arange(n[i] + 1) / (n[i] + 1))[:, None] * (path[i + 1] - path[i]) for i in range(L - 1)]
        out.append(path[-1:])
        return np.concatenate(out, 0).astype(np.float32)
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
    dev = paths.device
    d = torch.linalg.norm(paths[:, 1:] - paths[:, :-1], dim=-1)           # [P, W-1]
    n = torch.clamp(torch.ceil(d / resolution), min=1).to(torch.int64)    # [P, W-1]
    # segment (p, w) gives points t = k / n for k < n, the last one also t = 1
    cnt = n.clone()
    cnt[:, -1] += 1
    cnt = cnt.reshape(-1)
    seg = torch.repeat_interleave(torch.arange(cnt.numel(), device=dev), cnt)
    first = torch.cumsum(cnt, 0) - cnt
    k = torch.arange(seg.numel(), device=dev) - first[seg]
    t = k.to(paths.dtype) / n.reshape(-1)[seg].to(paths.dtype)
    p, w = seg // (W - 1), seg % (W - 1)
    a, b = paths[p, w], paths[p, w + 1]
    return a + t[:, None] * (b - a), p


def smooth_paths(paths: list, collision_context: dict, lower, upper, *, waypoints: int = 64, steps: int = 50,
                 lr: float = 0.05, margin: float = 0.02, beta: float = 50.0, w_len: float = 1.0,
                 resolution: float = 0.01, device=None):
    """Smooth each path (list of [L_i, dim] arrays) with projected gradient steps
    on the adjoint cost; re-validate at `resolution`; revert paths that fail.
    A path of at most `waypoints` vertices reverts to itself (resample_path keeps
    its vertices); for a longer one the reverted waypoints are its arc-length
    resampling, and `accepted` tells the caller to keep the original path.

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


class BatchSmoothContext:
    """Robot tables plus one world per path, resident on the device, for the
    batched adjoint (prrtc_b200_smooth_cost_grad_batch): path p is costed
    against collision_contexts[p]'s world and self pairs."""

    def __init__(self, collision_contexts, dim: int, margin: float = 0.02, beta: float = 50.0, w_len: float = 1.0,
                 device=None):
        from .prrtc import _pack_worlds

        self.lib = _lib.load()
        self.device = cuda_device(device)
        self.dim = int(dim)
        self.margin, self.beta, self.w_len = float(margin), float(beta), float(w_len)
        ctxs = list(collision_contexts)
        B = self.B = len(ctxs)
        self.robot_ctx = DeviceContext(ctxs[0], self.device, world_keys=False)
        packed, counts = _pack_worlds(ctxs, B)
        self.t = {}
        bi = _lib.BatchInputs()
        bi.batch = B
        bi.robot = self.robot_ctx.robot()
        for key in ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces", "self_pairs"):
            tab = torch.from_numpy(np.ascontiguousarray(packed[key])).to(self.device)
            cnt = torch.from_numpy(np.ascontiguousarray(counts[key], dtype=np.int32)).to(self.device)
            self.t[key], self.t[key + "_count"] = tab, cnt
            setattr(bi, key, tab.data_ptr() if tab.numel() else None)
            setattr(bi, "max_" + key, int(tab.shape[1]))
            setattr(bi, key + "_count", cnt.data_ptr())
        self.bi = bi
        self.ws = workspace(self.lib.prrtc_b200_smooth_batch_workspace_size(C.byref(bi)), self.device)

    def cost_grad(self, waypoints: torch.Tensor, need_grad: bool = True):
        wp = waypoints.detach().to(self.device, torch.float32).contiguous()
        P, W, dim = wp.shape
        if P != self.B:
            raise ValueError(f"expected {self.B} paths (one per world), got {P}")
        cost = torch.empty((P,), dtype=torch.float32, device=self.device)
        grad = torch.empty_like(wp) if need_grad else None
        _lib.check(self.lib.prrtc_b200_smooth_cost_grad_batch(C.byref(self.bi), dim, ptr(wp), W, self.margin,
                                                              self.beta, self.w_len, ptr(cost), ptr(grad),
                                                              self.ws.data_ptr(), self.ws.numel(), stream_handle()),
                   "prrtc_b200_smooth_cost_grad_batch")
        return cost, grad


def projected_steps(sctx, init: torch.Tensor, lower, upper, steps: int, lr: float) -> torch.Tensor:
    """`steps` projected gradient steps of the adjoint cost from `init` [P, W, dim]:
    endpoints fixed, joint limits enforced, step length lr per path (the
    gradient normalised per path)."""
    P, W, dim = init.shape
    lo = as_tensor(lower, torch.float32, init.device).reshape(1, 1, dim)
    hi = as_tensor(upper, torch.float32, init.device).reshape(1, 1, dim)
    x = init.clone()
    mask = torch.ones_like(x)
    mask[:, 0] = 0.0
    mask[:, -1] = 0.0
    for _ in range(steps):
        _, g = sctx.cost_grad(x)
        gn = torch.linalg.norm((g * mask).reshape(P, -1), dim=1).clamp_min(1e-12)
        x = torch.minimum(torch.maximum(x - lr * (g * mask) / gn[:, None, None], lo), hi)
    return x


def smooth_paths_batch(paths: list, collision_contexts: list, lower, upper, *, waypoints: int = 64,
                       steps: int = 50, lr: float = 0.05, margin: float = 0.02, beta: float = 50.0,
                       w_len: float = 1.0, resolution: float = 0.01, device=None):
    """smooth_paths for the paths of a batch plan, path p in its own world
    collision_contexts[p]: one batched adjoint launch per step for all paths,
    then exact re-validation of each smoothed path at `resolution` against its
    world; a path that fails reverts to its input.

    Returns (smoothed [P, waypoints, dim], accepted [P] bool, cost before [P],
    cost after [P])."""
    dev = cuda_device(device)
    dim = int(np.asarray(paths[0]).shape[1])
    init = torch.from_numpy(np.stack([resample_path(p, waypoints) for p in paths])).to(dev)
    sctx = BatchSmoothContext(collision_contexts, dim, margin, beta, w_len, dev)
    c0, _ = sctx.cost_grad(init, need_grad=False)
    x = projected_steps(sctx, init, lower, upper, steps, lr)
    c1, _ = sctx.cost_grad(x, need_grad=False)
    accepted = revalidate_batch(x, collision_contexts, resolution, dev)
    out = torch.where(accepted[:, None, None], x, init)
    return out, accepted, c0, c1


def revalidate_batch(paths: torch.Tensor, collision_contexts: list, resolution: float, device) -> torch.Tensor:
    """Exact binary re-validation of path p [W, dim] of `paths` at `resolution`
    against collision_contexts[p]; returns accepted [P] bool."""
    pts, owner = densify(paths, resolution)
    owner_np = owner.cpu().numpy()
    bounds = np.searchsorted(owner_np, np.arange(paths.shape[0] + 1))
    accepted = torch.ones((paths.shape[0],), dtype=torch.bool, device=device)
    for p, ctx in enumerate(collision_contexts):
        seg = pts[bounds[p]:bounds[p + 1]]
        if seg.shape[0]:
            v = CollisionChecker(ctx, paths.shape[2], "binary", 0.0, device).check(seg)
            accepted[p] = v.max() == 0
    return accepted
