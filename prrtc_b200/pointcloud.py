"""Environment point clouds: the point-cloud edge validation of the reference's
host-driven planner (``cuda-rrtc/jax/prrtc_robogpu.py``), on the SMs.

The reference validates candidate edges against an environment point cloud on
RT cores through an external OptiX checker
(``RoboGPUCollisionChecker.check_edges_collision_free``, called at
prrtc_robogpu.py:183-191), every point a sphere of radius ``r_env``.  Here the
cloud is hashed into a uniform grid on the device (``PointCloud``) and the
same sphere-vs-point test runs inside the collision checker, so it is
available in three places:

* ``PointCloudChecker.check_edges_collision_free`` -- the edge validator the
  host-driven loop calls (``prrtc_b200_check_edges``);
* ``prrtc_plan_robogpu`` -- that host-driven RRT-Connect loop itself
  (prrtc_robogpu.py:103-298), driving the edge validator;
* ``prrtc_plan(..., collision_context={..., "point_cloud": P, "r_env": r})``
  and ``prrtc_plan_batch`` -- the single-kernel planners with the cloud checked
  inside the kernel, which the reference cannot do (OptiX cannot be called
  from its planner kernel).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .device import DeviceContext, as_tensor, cuda_device, ptr, stream_handle, workspace
from .prrtc import PRRTCResult, _resolve_collision_mode

DEFAULT_CELL = 0.1  # about the largest robot sphere radius + r_env: <= 27 cells per query


class PointCloud:
    """Points [M, 3] hashed into a device grid (``prrtc_b200_point_cloud_build``).

    ``cell`` is the grid cell edge in metres; ``n_buckets`` (a power of two, 0 =
    next power of two >= M) the hash table size.  The grid lives in this
    object's workspace, so keep the object alive while it is used."""

    def __init__(self, points, r_env: float = 0.02, cell: float = DEFAULT_CELL, n_buckets: int = 0, device=None):
        self.lib = _lib.load()
        self.device = cuda_device(device)
        self.points = as_tensor(points, torch.float32, self.device, 3).contiguous()
        self.n = int(self.points.shape[0])
        self.r_env, self.cell = float(r_env), float(cell)
        self.ws = workspace(self.lib.prrtc_b200_point_cloud_workspace_size(self.n, int(n_buckets)), self.device)
        self.c = _lib.PointCloud()
        _lib.check(self.lib.prrtc_b200_point_cloud_build(ptr(self.points), self.n, self.cell, self.r_env,
                                                         int(n_buckets), self.ws.data_ptr(), self.ws.numel(),
                                                         C.byref(self.c), stream_handle()),
                   "prrtc_b200_point_cloud_build")

    def ref(self):
        return C.byref(self.c)

    def address(self) -> int:
        return C.addressof(self.c)


def cloud_from_context(ctx: Optional[dict], device) -> Optional[PointCloud]:
    """The PointCloud of a collision_context carrying ``point_cloud`` [M,3] (and
    optionally ``r_env``, ``point_cloud_cell``); None when it has none."""
    if ctx is None:
        return None
    pc = ctx.get("point_cloud")
    if pc is None:
        return None
    if isinstance(pc, PointCloud):
        return pc
    if np.asarray(pc.cpu() if torch.is_tensor(pc) else pc).reshape(-1, 3).shape[0] == 0:
        return None
    return PointCloud(pc, float(ctx.get("r_env", 0.02)), float(ctx.get("point_cloud_cell", DEFAULT_CELL)),
                      device=device)


class PointCloudChecker:
    """Edge validator over a robot's sphere model, world geometry and an
    optional point cloud: the role of ``RoboGPUCollisionChecker``."""

    def __init__(self, collision_context: dict, dim: int, collision_checker: str = "binary",
                 collision_margin: float = 0.02, device=None):
        self.lib = _lib.load()
        self.device = cuda_device(device)
        self.dim = int(dim)
        self.context = collision_context
        self.mode = _resolve_collision_mode(collision_checker)
        self.margin = float(collision_margin)
        self.ctx = DeviceContext(collision_context, self.device)
        self._cloud_key = None
        self._cloud: Optional[PointCloud] = None

    def _cloud_for(self, point_cloud, r_env: float) -> Optional[PointCloud]:
        if point_cloud is None:
            return None
        if isinstance(point_cloud, PointCloud):
            return point_cloud
        # like the reference, the grid is cached on the array's identity
        key = (id(point_cloud), float(r_env))
        if key != self._cloud_key:
            self._cloud = PointCloud(point_cloud, r_env, device=self.device)
            self._cloud_key = key
        return self._cloud

    def check_edges_collision_free(self, edges, world_geom: Optional[dict] = None, point_cloud=None,
                                   r_env: float = 0.02) -> torch.Tensor:
        """edges [S, G, dim] -> int32 [S], 1 where every waypoint is free."""
        e = as_tensor(edges, torch.float32, self.device).contiguous()
        if e.ndim != 3 or e.shape[2] != self.dim:
            raise ValueError(f"edges must have shape (S, G, {self.dim}), got {tuple(e.shape)}")
        S, G = int(e.shape[0]), int(e.shape[1])
        out = torch.empty((S,), dtype=torch.int32, device=self.device)
        if S == 0:
            return out
        ctx = self.ctx if world_geom is None else DeviceContext({**self.context, **world_geom}, self.device)
        robot, world = ctx.robot(), ctx.world()
        cloud = self._cloud_for(point_cloud, r_env)
        ws = workspace(self.lib.prrtc_b200_check_edges_workspace_size(C.byref(robot), C.byref(world), S, G),
                       self.device)
        _lib.check(self.lib.prrtc_b200_check_edges(C.byref(robot), C.byref(world),
                                                   cloud.ref() if cloud is not None else None, self.dim,
                                                   e.data_ptr(), S, G, self.mode, self.margin, out.data_ptr(),
                                                   ws.data_ptr(), ws.numel(), stream_handle()),
                   "prrtc_b200_check_edges")
        return out


# ----------------------------------------------------------------------------- host-driven planner

def _steer(q_from, q_to, step_size):
    """prrtc_robogpu.py:36-45."""
    delta = q_to - q_from
    dist = np.linalg.norm(delta, axis=1, keepdims=True)
    return q_from + delta * np.minimum(1.0, step_size / np.maximum(dist, 1e-8))


def _edge_waypoints(q_a, q_b, granularity):
    """prrtc_robogpu.py:48-59: G waypoints with both endpoints included."""
    ts = np.linspace(0.0, 1.0, granularity, dtype=np.float32)
    return (q_a[:, None, :] * (1.0 - ts)[None, :, None] + q_b[:, None, :] * ts[None, :, None]).astype(np.float32)


class _Tree:
    """Host tree of the host-driven planner (prrtc_robogpu.py:62-101)."""

    def __init__(self, root, max_nodes, dim):
        self.configs = np.zeros((max_nodes, dim), np.float32)
        self.parents = np.full((max_nodes,), -1, np.int32)
        self.configs[0], self.parents[0], self.size = root, 0, 1

    def add(self, q, parent):
        if self.size >= self.configs.shape[0]:
            return -1
        i = self.size
        self.configs[i], self.parents[i] = q, parent
        self.size += 1
        return i

    @property
    def view(self):
        return self.configs[: self.size]

    def nearest(self, queries):
        d2 = ((self.view[:, None, :] - queries[None, :, :]) ** 2).sum(-1)
        return np.argmin(d2, axis=0)

    def path_to(self, node):
        chain, cur = [], int(node)
        for _ in range(self.size):
            chain.append(self.configs[cur])
            p = int(self.parents[cur])
            if p == cur:
                break
            cur = p
        chain.reverse()
        return chain


def prrtc_plan_robogpu(start_config, goal_configs, robot: dict, robogpu_checker: PointCloudChecker,
                       world_geom: Optional[dict] = None, point_cloud=None, r_env: float = 0.02,
                       max_iterations: int = 5_000, step_size: float = 0.5, num_new_samples: int = 128,
                       granularity: int = 16, max_nodes: int = 1_000_000, connect_max_steps: int = 32,
                       min_vals=None, max_vals=None, seed: int = 0) -> PRRTCResult:
    """Host-driven RRT-Connect validated by the point-cloud edge checker
    (prrtc_robogpu.py:103-298): per iteration, ``num_new_samples`` uniform
    samples extend the active tree (one batched edge check), then a greedy
    connect of the other tree toward every new node (one batched check per
    step).  ``robot`` is the collision_context the checker was built from."""
    start = np.asarray(start_config, np.float32).reshape(-1)
    dim = start.shape[0]
    goals = np.asarray(goal_configs, np.float32).reshape(-1, dim)
    lo = np.asarray(min_vals if min_vals is not None else np.full(dim, -np.pi), np.float32)
    hi = np.asarray(max_vals if max_vals is not None else np.full(dim, np.pi), np.float32)
    rng = np.random.default_rng(seed)
    tree_a, tree_b = _Tree(start, max_nodes, dim), _Tree(goals[0], max_nodes, dim)
    cloud = robogpu_checker._cloud_for(point_cloud, r_env)

    def edges_free(qa, qb):
        if qa.shape[0] == 0:
            return np.zeros((0,), bool)
        f = robogpu_checker.check_edges_collision_free(_edge_waypoints(qa, qb, granularity), world_geom, cloud,
                                                       r_env)
        return f.cpu().numpy() == 1

    solved, connection, iterations = False, None, 0
    active, other = tree_a, tree_b
    for iterations in range(1, max_iterations + 1):
        samples = rng.uniform(lo, hi, size=(num_new_samples, dim)).astype(np.float32)
        near = active.nearest(samples)
        q_near = active.view[near]
        q_new = _steer(q_near, samples, step_size).astype(np.float32)
        new_nodes, new_cfg = [], []
        for s in np.nonzero(edges_free(q_near, q_new))[0]:
            idx = active.add(q_new[s], int(near[s]))
            if idx < 0:
                break
            new_nodes.append(idx)
            new_cfg.append(q_new[s])
        if not new_nodes:
            active, other = other, active
            continue
        targets = np.stack(new_cfg)
        ids = np.asarray(new_nodes, np.int32)
        oidx = other.nearest(targets)
        live = np.ones(targets.shape[0], bool)
        for _ in range(connect_max_steps):
            if not live.any():
                break
            li = np.nonzero(live)[0]
            q_from = other.view[oidx[li]]
            q_step = _steer(q_from, targets[li], step_size).astype(np.float32)
            ok = edges_free(q_from, q_step)
            for k, s in enumerate(li):
                if not ok[k]:
                    live[s] = False
                    continue
                idx = other.add(q_step[k], int(oidx[s]))
                if idx < 0:
                    live[s] = False
                    continue
                oidx[s] = idx
                if np.linalg.norm(q_step[k] - targets[s]) <= step_size * 1e-3 + 1e-6:
                    live[s] = False
                    a_node, b_node = int(ids[s]), idx
                    connection = (a_node, b_node) if active is tree_a else (b_node, a_node)
                    solved = True
                    break
            if solved:
                break
        if solved:
            break
        active, other = other, active

    path, cost = None, float("inf")
    if solved:
        pa = tree_a.path_to(connection[0])
        pb = tree_b.path_to(connection[1])
        pb.reverse()
        full = np.stack(pa + pb)
        path = torch.from_numpy(full)
        cost = float(np.linalg.norm(np.diff(full, axis=0), axis=1).sum())
    return PRRTCResult(solved=solved, path=path, tree_a_size=tree_a.size, tree_b_size=tree_b.size,
                       iterations=iterations, cost=cost, kernel_time_ms=None,
                       tree_a_configs=torch.from_numpy(tree_a.configs[: tree_a.size].T.copy()),
                       tree_b_configs=torch.from_numpy(tree_b.configs[: tree_b.size].T.copy()),
                       tree_a_parents=torch.from_numpy(tree_a.parents[: tree_a.size].copy()),
                       tree_b_parents=torch.from_numpy(tree_b.parents[: tree_b.size].copy()))
