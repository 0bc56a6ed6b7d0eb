"""Batched collision checking, forward kinematics and Halton sampling on the GPU.

These expose the planner's own device code as stand-alone primitives: the
checker the planner runs on every edge waypoint (the reference's checkers,
cuda-rrtc/CUDA/prrtc_planner.cu:234-655), its FK, and its per-explorer Halton
sampler (144-157, 747-788).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import DeviceContext, as_tensor, cuda_device, ptr, stream_handle, workspace
from .prrtc import _resolve_collision_mode


class CollisionChecker:
    """A collision context resident on the GPU, reusable across calls.  A
    context with a ``point_cloud`` entry [M,3] (and ``r_env``) is checked
    against the cloud too."""

    def __init__(self, collision_context: dict, dim: int, collision_checker: str = "binary",
                 collision_margin: float = 0.02, device=None):
        self.lib = _lib.load()
        self.device = cuda_device(device)
        self.ctx = DeviceContext(collision_context, self.device)
        self.dim = int(dim)
        self.mode = _resolve_collision_mode(collision_checker)
        self.margin = float(collision_margin)
        self._robot = self.ctx.robot()
        self._world = self.ctx.world()
        self.ws = workspace(self.lib.prrtc_b200_check_configs_workspace_size(C.byref(self._robot),
                                                                           C.byref(self._world)), self.device)
        from .pointcloud import cloud_from_context

        self.cloud = cloud_from_context(collision_context, self.device)

    def check(self, configs, full_sweep: bool = False, out: torch.Tensor | None = None,
              stream: torch.cuda.Stream | None = None) -> torch.Tensor:
        """int32 verdicts [n] (1 = in collision) for configurations [n, dim]."""
        cf = as_tensor(configs, torch.float32, self.device).reshape(-1, self.dim)
        n = int(cf.shape[0])
        if out is None:
            out = torch.empty((n,), dtype=torch.int32, device=self.device)
        if self.cloud is not None:  # one-waypoint edges through the edge checker, which sees the cloud
            free = torch.empty((n,), dtype=torch.int32, device=self.device)
            ws = workspace(self.lib.prrtc_b200_check_edges_workspace_size(C.byref(self._robot), C.byref(self._world),
                                                                         n, 1), self.device)
            _lib.check(self.lib.prrtc_b200_check_edges(C.byref(self._robot), C.byref(self._world), self.cloud.ref(),
                                                       self.dim, ptr(cf), n, 1, self.mode, self.margin, ptr(free),
                                                       ws.data_ptr(), ws.numel(), stream_handle(stream)),
                       "prrtc_b200_check_edges")
            torch.sub(1, free, out=out)
            return out
        _lib.check(self.lib.prrtc_b200_check_configs(C.byref(self._robot), C.byref(self._world), self.dim, ptr(cf),
                                                     n, self.mode, self.margin, 1 if full_sweep else 0, ptr(out),
                                                     self.ws.data_ptr(), self.ws.numel(), stream_handle(stream)),
                   "prrtc_b200_check_configs")
        return out

    def __call__(self, configs) -> np.ndarray:
        return self.check(configs).cpu().numpy()


def check_configs(configs, collision_context: dict, collision_checker: str = "binary",
                  collision_margin: float = 0.02, full_sweep: bool = False, device=None) -> torch.Tensor:
    cf = torch.as_tensor(np.asarray(configs) if not isinstance(configs, torch.Tensor) else configs)
    dim = int(cf.shape[-1])
    return CollisionChecker(collision_context, dim, collision_checker, collision_margin, device).check(
        cf, full_sweep=full_sweep)


def forward_kinematics(configs, collision_context: dict, device=None) -> torch.Tensor:
    """Link frames [n, n_joints, 12] (row-major R, then t) in output frame order."""
    lib = _lib.load()
    dev = cuda_device(device)
    ctx = DeviceContext(collision_context, dev, world_keys=False)
    cf = as_tensor(configs, torch.float32, dev)
    dim = int(cf.shape[-1])
    cf = cf.reshape(-1, dim)
    J = ctx.n("fk_parent_idx")
    out = torch.empty((cf.shape[0], J, 12), dtype=torch.float32, device=dev)
    r = ctx.robot()
    _lib.check(lib.prrtc_b200_fk(C.byref(r), dim, ptr(cf), int(cf.shape[0]), ptr(out), stream_handle()),
               "prrtc_b200_fk")
    return out


def halton_samples(explorer: int, n: int, min_vals, max_vals, device=None) -> torch.Tensor:
    """First n samples [n, dim] of explorer `explorer`'s Halton stream."""
    lib = _lib.load()
    dev = cuda_device(device)
    lo = as_tensor(min_vals, torch.float32, dev).reshape(-1)
    hi = as_tensor(max_vals, torch.float32, dev).reshape(-1)
    dim = int(lo.shape[0])
    out = torch.empty((n, dim), dtype=torch.float32, device=dev)
    _lib.check(lib.prrtc_b200_halton(int(explorer), int(n), dim, ptr(lo), ptr(hi), ptr(out), stream_handle()),
               "prrtc_b200_halton")
    return out


def gpu_checker(device=None):
    """A ``checker(configs, ctx) -> verdicts`` callable for the scene generators."""
    cache: dict = {}

    def _check(configs, ctx):
        key = id(ctx)
        if key not in cache:
            cache.clear()
            cache[key] = (ctx, CollisionChecker(ctx, int(np.asarray(configs).shape[-1]), device=device))
        return cache[key][1](configs)

    return _check
